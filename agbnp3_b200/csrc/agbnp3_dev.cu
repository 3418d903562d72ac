/*
 * AGBNP3 energy + gradient on the GPU.
 *
 * One evaluation of the reference's agbnp3_total_energy()
 * (agbnp3.c:1221-1816) as a fixed sequence of kernels over a device system
 * of one or more concatenated instances:
 *
 *   prep      gather coordinates to internal order, reset accumulators
 *   nblist    heavy-atom near list via a hashed cell grid: count -> scan ->
 *             emit, each list sorted by (float d^2, index)  (agbnp3.c:3978-4115)
 *   volumes   overlap tree, orders 2..5, level-synchronous count -> scan ->
 *             emit; kept overlaps are stored once and reused by the
 *             derivative pass  (agbnp3_cpu_simd_kernels.c:1064-1598)
 *   scaling   scaling factors, filtered areas, cavity energy
 *             (agbnp3_utils.c:524-613)
 *   invb      descreening integrals -> inverse Born radii -> Born radii,
 *             vdW energy  (agbnp3_cpu_simd_kernels.c:500-678,
 *             agbnp3_utils.c:615-670, agbnp3.c:1466-1487)
 *   agb       GB pair energy, gradient at constant Born radii, A_i
 *             (agbnp3_cpu_simd_kernels.c:66-151, 329-460)
 *   gbders    gradient through the Born radii at constant self volumes and
 *             U_i / V_i  (agbnp3_cpu_simd_kernels.c:681-904)
 *   ws        water sites, free volumes, HB energy and gradient
 *             (agbnp3.c:1837-3761, agbnp3_cpu_simd_kernels.c:2637-2954)
 *   treeders  self-volume and surface-area derivatives over every kept
 *             overlap  (agbnp3_cpu_simd_kernels.c:1601-2405)
 *   final     outputs to caller order, per-instance energy sums
 *
 * The pair and overlap arithmetic is templated on R: double for the plain
 * FP64 path, float for the mixed path.  Every accumulation (Born-radius
 * descreening sums, inclusion-exclusion volume and area sums, gradients,
 * energies) is double in both.  No index is ever produced by an atomic:
 * sizes come from count -> exclusive scan -> emit.
 */
#include "agbnp3_launch.cuh"
#include "agbnp3_dev.h"

#include <cuda_bf16.h>

#include <cmath>
#include <dlfcn.h>
#include <nccl.h>
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* model constants (agbnp3_private.h:88-137, 680-684; agbnp3.c:1230-1235) */
#define C_PI 3.14159265359
#define C_KFC 2.5
#define C_PFC 2.97354
#define C_VOLA 0.01
#define C_VOLB 0.1
#define C_RINC 0.5
#define C_HBRAD 1.4
#define C_HBLEN 2.5
#define C_HBSWA 0.65
#define C_HBSWB 1.0
#define C_HBSWA0 0.6
#define C_RW 1.4
#define C_TOKCAL 332.0
#define C_AMAX 20.0

#define BLK 128
#define FULLMASK 0xffffffffu

struct __align__(16) f4 {
  float x, y, z, w;
};

/* ------------------------------------------------------------------------ */
/* device view: every pointer a kernel may need                             */
/* ------------------------------------------------------------------------ */
struct View {
  int ninst, natoms, nws, ntypes, compat;
  const int *inst_begin, *inst_nheavy, *inst_of, *ws_begin, *ws_inst;
  const double *inst_df;
  const float *inst_cell;
  const int *bucket_begin, *bucket_mask;
  const int *ext_of;
  const double *r, *charge, *igamma, *sgamma, *ialpha, *salpha, *vols;
  const int *rtype;
  const int *ws_kind, *ws_parent, *ws_nparent, *ws_prev;
  const double *ws_khb;
  /* per evaluation */
  const double *x_ext, *y_ext, *z_ext;
  f4 *pos;
  double *pxd, *pyd, *pzd;
  int *atom_cell, *atom_bucket;
  int *bucket_count, *bucket_start, *bucket_cursor;
  f4 *cell_pos;  /* per bucket slot: the atom's position and radius */
  int2 *cell_id; /* per bucket slot: the atom and its packed cell */
  int *nl_count, *nl_off, *nl_list;
  int slab_w;            /* near partners an (atom, neighbour cell) sub-slab holds */
  int nl_cells;          /* near-list search by k_nl_cells (large systems) instead of k_nl_c27 */
  int *slab_j;           /* [natoms * 27 * slab_w] partners, unordered */
  float *slab_d2;        /* [natoms * 27 * slab_w] their float d^2 */
  float *nl_d2;
  int cap_nl;
  int cap[AGB_MAX_ORDER + 1];
  int *lv_cnt[AGB_MAX_ORDER + 1], *lv_off[AGB_MAX_ORDER + 1];
  unsigned long long *lv_mask[AGB_MAX_ORDER + 1]; /* kept siblings of each generating overlap */
  int *lv_own[AGB_MAX_ORDER + 1];                 /* generating overlap of each record */
  int *par[AGB_MAX_ORDER + 1], *gend[AGB_MAX_ORDER + 1];
  void *rec[AGB_MAX_ORDER + 1];
  int *dc; /* device counters, DC_* */
  double *volumep, *surf, *surf_f, *sp, *spe, *psvol, *gammap;
  double *bfil, *bder, *br, *brw, *dera, *q2ab, *abrw, *deru, *derv, *derh, *derus, *dervs;
  double *g_gb, *g_vw, *g_cav, *g_hb; /* [natoms*3], internal order */
  double *eatom;                      /* [7][natoms] */
  double *ews;                        /* [nws] */
  void *wpos, *wdpos;                 /* R[3*nws], R[36*nws] */
  void *tdat;                         /* TdAtom<R>[natoms]: what the tree-derivative pass reads per parent */
  double *wsp;                        /* [nws] */
  double *o_sp, *o_br, *o_sa, *o_gb, *o_gv, *o_gc, *o_gh;
  int nbuckets;
  void *pa[12];      /* packed operands (R[natoms] each); the pair-stage ones in slot order */
  /* pair-stage slot order: each instance's heavy atoms, then its hydrogens,
     each group sorted along a Hilbert curve so that 32 consecutive slots
     are a compact cluster (identity until the first evaluation sets it) */
  const int *slot_atom, *atom_slot;
  int *slot_type; /* radius type by slot */
  int *slot_hvcol; /* by slot: offset (hvslot[type] * AGB_NA) of the type's column of the shared tables */
  /* Verlet-skin reuse of the near list (skin > 0): candidates j > g within
     the near-list cutoff plus the skin, grouped by atom (CSR cand_off /
     cand_cnt), the positions they were built from, and per candidate the
     exact near-list flag and its exclusive scan */
  float skin;
  int cap_cand;
  int *cand_j, *cand_own, *cand_flag, *cand_scan, *cand_off, *cand_cnt;
  f4 *pos_ref;
  int *nl_c27, *nl_o27; /* near-list counts / offsets per (atom, neighbour cell) */
  int *nl_tmp, *nl_own; /* unsorted entries and their atom */
  int *ws_c27, *ws_o27, *ws_cand; /* water-site candidates per (site, cell) */
  int *ws_srt;                    /* the same candidates in index order */
  int cap_wsc;
  double *acc_beta; /* descreening sums */
  /* per 32-slot tile of the pair slots: float bounding box of the positions
     (lo x, y, z, smallest 1/(hR)) and (hi x, y, z, 0), rounded outward */
  float4 *tbox;
  /* learned surrogate: every atom's class (-1: none) and a hashed grid of
     SF_RC cells over all atoms of each instance (buckets sf_bbegin[I] ..
     + sf_bmask[I]; slots hold position + class and atom + cell key) */
  signed char *sclass;
  int sf_nbuckets;
  const int *sf_bbegin, *sf_bmask;
  int *sf_bcount, *sf_bstart, *sf_bcursor, *sf_abucket, *sf_dc;
  f4 *sf_spos;
  int2 *sf_sid;
  /* Q4 tables as per-interval cubics in t = a/h - k, c0..c3 */
  const float4 *tabv_f;
  const double4 *tabv_d;
  /* the FP32 tables whose descreener type has heavy atoms, as
     [descreened type][heavy slot of the descreener type][AGB_NA], and the
     heavy slot of each type (0 for a type only hydrogens have: its lookups
     all fall on the zero record AGB_NA-1, the same in every table) */
  const float4 *tabh_f;
  const int *hvslot;
  int nhv;
};

enum { DC_N = 0, DC_NB, DC_NWS, DC_NL, DC_ERR, DC_L0 /* DC_L0+m: kept of order m */, DC_C0 = DC_L0 + 8 /* scratch */,
       DC_W27 = DC_C0 + 2, DC_WSC,
       /* Verlet skin: rebuild flag of this evaluation, candidate scan length
          (27 N when rebuilding, else 0), that scan's total, the live
          candidates of the last build, builds so far */
       DC_REBUILD = DC_C0 + 8, DC_CLEN, DC_CTOT, DC_NCAND, DC_NBUILD,
       DC_SLABMAX /* near partners of the fullest overflowing (atom, cell) sub-slab */,
       DC_N27 /* 27 N */,
       DC_GBDQ /* next work item of the chain-rule pass (reset by k_agb_post) */,
       DC_DESQ /* next half item of the descreening pass (reset by k_pack_sp) */,
       DC_AGBQ /* next work item of the GB pair pass (reset by k_born) */ };
#define DC_SIZE (DC_C0 + 18)

/* record fields of a kept overlap, stored contiguously per record (12
   slots, three 4-wide vectors) */
/* a kept overlap's record: the product Gaussian (a, p, centre), its raw
   volume and the switch derivatives; the switched volume is used only when
   the overlap is made and is not stored */
enum { F_A = 0, F_P, F_CX, F_CY, F_CZ, F_GVOL, F_FP, F_FPP, F_NUM = 8 };

/* packed per-atom operands, in the working precision: position, 1/R,
   1/(h R), Gaussian exponent KFC/R^2, sp, charge, B, 1/B, q2ab, abrw.
   1/R and the exponent (the overlap tree's) are indexed by atom; the pair
   stages' operands by pair slot (View::atom_slot) */
enum { PA_X = 0, PA_Y, PA_Z, PA_RINV, PA_RH, PA_SP, PA_ALPHA, PA_Q, PA_B, PA_BINV, PA_Q2AB, PA_ABRW, PA_NUM };

template <typename R>
__device__ __forceinline__ R *pa(const View &v, int k) {
  return (R *)v.pa[k];
}

/* ------------------------------------------------------------------------ */
/* math helpers                                                             */
/* ------------------------------------------------------------------------ */
__device__ __forceinline__ float m_exp(float x) { return expf(x); }
__device__ __forceinline__ double m_exp(double x) { return exp(x); }
__device__ __forceinline__ float m_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double m_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float m_rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double m_rsqrt(double x) { return rsqrt(x); }

/* the pair passes' special functions: in FP32 the single-instruction PTX
   approximations (relative error near 2^-22, denormals flushed), in FP64
   the library functions */
__device__ __forceinline__ float p_sqrt(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double p_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float p_rsqrt(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double p_rsqrt(double x) { return rsqrt(x); }

/* reciprocal and exponential of the FP32 overlap arithmetic: approximations
   (rcp.approx, ex2.approx; relative error near 2^-22) in float, the exact
   operations in double */
__device__ __forceinline__ float f_rcp(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double f_rcp(double x) { return 1.0 / x; }
__device__ __forceinline__ float f_exp(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x * 1.4426950408889634f));
  return y;
}
__device__ __forceinline__ double f_exp(double x) { return exp(x); }

template <typename R>
__device__ __forceinline__ R px(const View &v, int g);
template <>
__device__ __forceinline__ float px<float>(const View &v, int g) { return v.pos[g].x; }
template <>
__device__ __forceinline__ double px<double>(const View &v, int g) { return v.pxd[g]; }
template <typename R>
__device__ __forceinline__ R py(const View &v, int g);
template <>
__device__ __forceinline__ float py<float>(const View &v, int g) { return v.pos[g].y; }
template <>
__device__ __forceinline__ double py<double>(const View &v, int g) { return v.pyd[g]; }
template <typename R>
__device__ __forceinline__ R pz(const View &v, int g);
template <>
__device__ __forceinline__ float pz<float>(const View &v, int g) { return v.pos[g].z; }
template <>
__device__ __forceinline__ double pz<double>(const View &v, int g) { return v.pzd[g]; }

__device__ __forceinline__ void set_err(const View &v, int bit) { atomicOr(&v.dc[DC_ERR], bit); }

/* quintic switch from 0 at xa to 1 at xb with first and second derivative
   (agbnp3.c:1120-1145, agbnp3_cpu_simd_kernels.c:2487-2529) */
template <typename R>
__device__ __forceinline__ R poly_switch(R x, R xa, R xb, R &fp, R &fpp) {
  if (x > xb) {
    fp = fpp = R(0);
    return R(1);
  }
  if (x < xa) {
    fp = fpp = R(0);
    return R(0);
  }
  R d = R(1) / (xb - xa), u = (x - xa) * d, u2 = u * u;
  fp = d * R(30) * u2 * (R(1) - R(2) * u + u2);
  fpp = d * d * R(60) * u * (R(1) - R(3) * u + R(2) * u2);
  return u * u2 * (R(10) - R(15) * u + R(6) * u2);
}

/* product of two Gaussians a1 p1 (x1) and a2 p2 (x2): exponent, prefactor,
   centre, raw overlap volume and the switched volume with its derivative
   factors (agbnp3_cpu_simd_kernels.c:2418-2477) */
template <typename R>
struct Ov {
  R a, p, cx, cy, cz, gvol, gvolp, fp, fpp;
};

template <typename R>
__device__ __forceinline__ Ov<R> ogauss(R a1, R p1, R x1, R y1, R z1, R a2, R p2, R x2, R y2, R z2) {
  Ov<R> o;
  R dx = x2 - x1, dy = y2 - y1, dz = z2 - z1;
  R d2 = dx * dx + dy * dy + dz * dz;
  o.a = a1 + a2;
  R inv = f_rcp(o.a);
  o.p = p1 * p2 * f_exp(-a1 * a2 * d2 * inv);
  R u = R(C_PI) * inv;
  o.gvol = o.p * u * p_sqrt(u);
  o.cx = inv * (a1 * x1 + a2 * x2);
  o.cy = inv * (a1 * y1 + a2 * y2);
  o.cz = inv * (a1 * z1 + a2 * z2);
  R sp, spp;
  R s = poly_switch<R>(o.gvol, R(C_VOLA), R(C_VOLB), sp, spp);
  o.gvolp = s * o.gvol;
  o.fp = s + o.gvol * sp;
  o.fpp = R(2) * sp + o.gvol * spp;
  return o;
}

template <typename R>
__device__ __forceinline__ bool kept(R gvolp) {
  return gvolp > R(FLT_MIN);
}

/* ------------------------------------------------------------------------ */
/* prep: gather coordinates into internal order, reset accumulators         */
/* ------------------------------------------------------------------------ */
__global__ void k_prep(View v) {
  AGB_GRID_STRIDE(g, v.natoms) {
    int e = v.ext_of[g];
    double x = v.x_ext[e], y = v.y_ext[e], z = v.z_ext[e], r = v.r[g];
    f4 p;
    p.x = (float)x;
    p.y = (float)y;
    p.z = (float)z;
    p.w = (float)r;
    v.pos[g] = p;
    v.pxd[g] = x;
    v.pyd[g] = y;
    v.pzd[g] = z;
    int I = v.inst_of[g];
    bool heavy = g < v.inst_begin[I] + v.inst_nheavy[I];
    v.volumep[g] = heavy ? v.vols[g] : 0.0;
    v.surf[g] = heavy ? 4.0 * C_PI * r * r : 0.0;
    v.dera[g] = v.deru[g] = v.derv[g] = v.derh[g] = 0.0;
    for (int c = 0; c < 3; c++) {
      v.g_gb[3 * g + c] = v.g_vw[3 * g + c] = v.g_cav[3 * g + c] = v.g_hb[3 * g + c] = 0.0;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* nblist: hashed cell grid over the heavy atoms of each instance           */
/* ------------------------------------------------------------------------ */
__device__ __forceinline__ int cell_hash(int cx, int cy, int cz, int mask) {
  unsigned h = (unsigned)cx * 73856093u ^ (unsigned)cy * 19349663u ^ (unsigned)cz * 83492791u;
  return (int)(h & (unsigned)mask);
}

/* 10 bits per axis: the 27 cells around any cell have distinct keys, and a
   far cell sharing a key holds only atoms beyond every cutoff */
__device__ __forceinline__ int cell_key(int cx, int cy, int cz) {
  return (cx & 1023) | ((cy & 1023) << 10) | ((cz & 1023) << 20);
}

__device__ __forceinline__ void cell_of(float x, float y, float z, float inv, int &cx, int &cy, int &cz) {
  cx = (int)floorf(x * inv);
  cy = (int)floorf(y * inv);
  cz = (int)floorf(z * inv);
}

__global__ void k_cell_count(View v) {
  AGB_GRID_STRIDE(g, v.natoms) {
    int I = v.inst_of[g];
    if (g >= v.inst_begin[I] + v.inst_nheavy[I]) {
      /* hydrogens have no near list: their per-direction counts are zero
         (the near-list search writes those of the heavy atoms) */
      if (v.nl_cells && v.skin <= 0.0f)
        for (int c = 0; c < 27; c++) v.nl_c27[27 * g + c] = 0;
      continue;
    }
    float inv = 1.0f / v.inst_cell[I];
    f4 p = v.pos[g];
    int cx, cy, cz;
    cell_of(p.x, p.y, p.z, inv, cx, cy, cz);
    v.atom_cell[3 * g] = cx;
    v.atom_cell[3 * g + 1] = cy;
    v.atom_cell[3 * g + 2] = cz;
    int b = v.bucket_begin[I] + cell_hash(cx, cy, cz, v.bucket_mask[I]);
    v.atom_bucket[g] = b;
    atomicAdd(&v.bucket_count[b], 1);
  }
}

__global__ void k_cell_fill(View v) {
  AGB_GRID_STRIDE(g, v.natoms) {
    int I = v.inst_of[g];
    if (g >= v.inst_begin[I] + v.inst_nheavy[I]) continue;
    int b = v.atom_bucket[g];
    /* slot order inside a bucket is arbitrary; every consumer sorts */
    int s = v.bucket_start[b] + atomicAdd(&v.bucket_cursor[b], 1);
    v.cell_pos[s] = v.pos[g];
    v.cell_id[s] = make_int2((int)g, cell_key(v.atom_cell[3 * g], v.atom_cell[3 * g + 1], v.atom_cell[3 * g + 2]));
  }
}

/* the reference's float membership test d^2 < (1.6 (ri + rj))^2, evaluated
   without fused operations (agbnp3.c:4041-4049) */
__device__ __forceinline__ bool near_test(const f4 &a, const f4 &b, float &d2) {
  float dx = __fsub_rn(b.x, a.x), dy = __fsub_rn(b.y, a.y), dz = __fsub_rn(b.z, a.z);
  d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
  float u = __fmul_rn(__fadd_rn(a.w, b.w), 1.6f);
  return d2 < __fmul_rn(u, u);
}

/* the heavy atoms of instance I in cell (ax, ay, az): fn(j, position of j)
   once each; a bucket's slots are contiguous records */
template <typename Fn>
__device__ __forceinline__ void for_cell(const View &v, int I, int ax, int ay, int az, Fn fn) {
  int b = v.bucket_begin[I] + cell_hash(ax, ay, az, v.bucket_mask[I]);
  int s0 = v.bucket_start[b], s1 = s0 + v.bucket_count[b];
  const int key = cell_key(ax, ay, az);
  for (int s = s0; s < s1; s++) {
    int2 id = v.cell_id[s];
    f4 p = v.cell_pos[s];
    if (id.y == key) fn(id.x, p);
  }
}

/* one thread per (heavy atom, neighbour cell), taken direction-major over
   the pair slots (a warp's atoms are spatially close and look into the
   same neighbour direction): the atom's partners j > i in that cell that
   pass the near test go to the (atom, cell) sub-slab of slab_w entries,
   their number to nl_c27.  No atomics: every entry and count has one
   writer.  An overflowing sub-slab sets the error word and the largest
   count needed. */
__global__ void k_nl_c27(View v) {
  AGB_GRID_STRIDE(q, 27LL * v.natoms) {
    const int c = (int)(q / v.natoms), g = v.slot_atom[(int)(q % v.natoms)];
    const int I = v.inst_of[g];
    int cnt = 0;
    if (g < v.inst_begin[I] + v.inst_nheavy[I]) {
      const f4 a = v.pos[g];
      const size_t base = ((size_t)g * 27 + c) * v.slab_w;
      for_cell(v, I, v.atom_cell[3 * g] + c % 3 - 1, v.atom_cell[3 * g + 1] + (c / 3) % 3 - 1,
               v.atom_cell[3 * g + 2] + c / 9 - 1, [&](int j, const f4 &b) {
                 float d2;
                 if (j > g && near_test(a, b, d2)) {
                   if (cnt < v.slab_w) {
                     v.slab_j[base + cnt] = j;
                     v.slab_d2[base + cnt] = d2;
                   }
                   cnt++;
                 }
               });
      if (cnt > v.slab_w) {
        set_err(v, AGB_ERR_NL_CAP);
        atomicMax(&v.dc[DC_SLABMAX], cnt); /* capacity statistic of the error path */
      }
    }
    v.nl_c27[27 * g + c] = cnt;
  }
}

/* the near-list search over the cell grid's slots: a warp takes 32
   consecutive slots (heavy atoms, grouped by bucket, so mostly one or two
   cells) and one neighbour-cell direction; its lanes are those atoms.  The
   lanes that look into the same neighbour bucket walk its slots together
   (the same slot on every lane, one broadcast load), each testing the slot's
   atom against its own: the pairs j > i passing the near test go to the
   lane's (atom, direction) sub-slab of slab_w entries and their number to
   nl_c27[27 i + c].  No atomics: every entry and count has one writer.  An
   overflowing sub-slab sets the error word and the largest count needed.
   The counts of hydrogens (not in the grid) are cleared by k_cell_count. */
__global__ void k_nl_cells(View v) {
  const int nslot = v.dc[DC_C0 + 7]; /* heavy atoms in the grid */
  const int nchunk = (nslot + 31) >> 5;
  const int lane = threadIdx.x & 31;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long q = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < 27LL * nchunk; q += nw) {
    const int c = (int)(q / nchunk), s = (int)(q % nchunk) * 32 + lane;
    const bool valid = s < nslot;
    int g = 0, bB = -1, keyB = 0, cnt = 0;
    f4 a = {0.f, 0.f, 0.f, 0.f};
    if (valid) {
      g = v.cell_id[s].x;
      a = v.cell_pos[s];
      const int I = v.inst_of[g];
      const int ax = v.atom_cell[3 * g] + c % 3 - 1, ay = v.atom_cell[3 * g + 1] + (c / 3) % 3 - 1,
                az = v.atom_cell[3 * g + 2] + c / 9 - 1;
      bB = v.bucket_begin[I] + cell_hash(ax, ay, az, v.bucket_mask[I]);
      keyB = cell_key(ax, ay, az);
    }
    const size_t base = ((size_t)g * 27 + c) * v.slab_w;
    unsigned todo = __ballot_sync(0xffffffffu, valid);
    while (todo) {
      const int leader = __ffs(todo) - 1;
      const int b = __shfl_sync(0xffffffffu, bB, leader), key = __shfl_sync(0xffffffffu, keyB, leader);
      const bool mine = valid && bB == b && keyB == key;
      todo &= ~__ballot_sync(0xffffffffu, mine);
      const int s0 = v.bucket_start[b], s1 = s0 + v.bucket_count[b];
#pragma unroll 4
      for (int t = s0; t < s1; t++) {
        const int2 id = v.cell_id[t];
        const f4 p = v.cell_pos[t];
        float d2;
        if (mine && id.y == key && id.x > g && near_test(a, p, d2)) {
          if (cnt < v.slab_w) {
            v.slab_j[base + cnt] = id.x;
            v.slab_d2[base + cnt] = d2;
          }
          cnt++;
        }
      }
    }
    if (valid) {
      if (cnt > v.slab_w) {
        set_err(v, AGB_ERR_NL_CAP);
        atomicMax(&v.dc[DC_SLABMAX], cnt); /* capacity statistic of the error path */
      }
      v.nl_c27[27 * g + c] = cnt;
    }
  }
}

/* each atom's list in (float d^2, index) order (agbnp3.c:3766-3792,
   4062-4066), one warp per atom: lane c < 27 copies its cell's sub-slab to
   the warp's buffer in shared memory (to the atom's range of the list in
   global memory when it holds more than NLR_BUF entries), at the place the
   warp's scan of the per-cell counts gives, then every entry is written at
   its rank; the list starts where the scan of all counts places it */
#define NLR_BUF 64 /* near-list entries of an atom ranked in shared memory */
__global__ void k_nl_rank27(View v) {
  if (v.dc[DC_ERR] & AGB_ERR_NL_CAP) return;
  __shared__ int sj[BLK / 32][NLR_BUF];
  __shared__ float sd[BLK / 32][NLR_BUF];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long g = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < v.natoms; g += nw) {
    const int cnt = lane < 27 ? v.nl_c27[27 * g + lane] : 0;
    int x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULLMASK, x, o);
      if (lane >= o) x += y;
    }
    const int m = __shfl_sync(FULLMASK, x, 31), o = v.nl_o27[27 * g];
    if (lane == 0) {
      v.nl_off[g] = o;
      v.nl_count[g] = m;
    }
    if (m == 0) continue;
    if (o + m > v.cap_nl) {
      if (lane == 0) set_err(v, AGB_ERR_NL_CAP);
      continue;
    }
    const size_t sb = ((size_t)g * 27 + lane) * v.slab_w;
    if (m <= NLR_BUF) { /* the usual case: the atom's entries in shared memory */
      for (int k = 0; k < cnt; k++) {
        sj[wp][x - cnt + k] = v.slab_j[sb + k];
        sd[wp][x - cnt + k] = v.slab_d2[sb + k];
      }
      __syncwarp();
      for (int k = lane; k < m; k += 32) {
        const float d2 = sd[wp][k];
        const int j = sj[wp][k];
        int rank = 0;
        for (int b = 0; b < m; b++) {
          const float db = sd[wp][b];
          rank += (db < d2) || (db == d2 && sj[wp][b] < j);
        }
        v.nl_list[o + rank] = j;
        v.nl_own[o + rank] = (int)g;
      }
      __syncwarp(); /* the buffer is read before the next atom fills it */
      continue;
    }
    for (int k = 0; k < cnt; k++) {
      v.nl_tmp[o + x - cnt + k] = v.slab_j[sb + k];
      v.nl_d2[o + x - cnt + k] = v.slab_d2[sb + k];
    }
    __syncwarp();
    for (int k = lane; k < m; k += 32) {
      const float d2 = v.nl_d2[o + k];
      const int j = v.nl_tmp[o + k];
      int rank = 0;
      for (int b = 0; b < m; b++) {
        const float db = v.nl_d2[o + b];
        rank += (db < d2) || (db == d2 && v.nl_tmp[o + b] < j);
      }
      v.nl_list[o + rank] = j;
      v.nl_own[o + rank] = (int)g;
    }
  }
}

/* ---- Verlet skin ------------------------------------------------------ */
/* The near list of an evaluation is exactly the cell-grid one: candidates
   are the pairs within 1.6 (ri + rj) + skin when they were searched, and
   while no heavy atom has moved skin/2 from those positions every pair now
   within 1.6 (ri + rj) is among them; the reference's float test is
   applied to the candidates at the current positions. */

/* any heavy atom at skin/2 or more from its build position (or a build
   forced by unset positions) sets the rebuild flag */
__global__ void k_skin_check(View v) {
  const float lim = 0.5f * v.skin * 0.9999f;
  AGB_GRID_STRIDE(g, v.natoms) {
    int I = v.inst_of[g];
    if (g >= v.inst_begin[I] + v.inst_nheavy[I]) continue;
    f4 p = v.pos[g], q = v.pos_ref[g];
    float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
    if (!(dx * dx + dy * dy + dz * dz < lim * lim)) v.dc[DC_REBUILD] = 1;
  }
}

__global__ void k_skin_len(View v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int rb = v.dc[DC_REBUILD];
    v.dc[DC_CLEN] = rb ? 27 * v.natoms : 0;
    if (rb) v.dc[DC_NBUILD] += 1;
  }
}

__device__ __forceinline__ bool cand_test(const f4 &a, const f4 &b, float skin) {
  float dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
  float u = 1.6f * (a.w + b.w) + skin + 1e-3f;
  return dx * dx + dy * dy + dz * dz < u * u;
}

/* one thread per (heavy atom, neighbour cell), only when rebuilding */
__global__ void k_cand_count27(View v) {
  if (!v.dc[DC_REBUILD]) return;
  AGB_GRID_STRIDE(q, 27LL * v.natoms) {
    int g = (int)(q / 27), c = (int)(q % 27);
    int I = v.inst_of[g];
    int cnt = 0;
    if (g < v.inst_begin[I] + v.inst_nheavy[I]) {
      f4 a = v.pos[g];
      for_cell(v, I, v.atom_cell[3 * g] + c % 3 - 1, v.atom_cell[3 * g + 1] + (c / 3) % 3 - 1,
               v.atom_cell[3 * g + 2] + c / 9 - 1, [&](int j, const f4 &b) {
                 if (j > g && cand_test(a, b, v.skin)) cnt++;
               });
    }
    v.nl_c27[q] = cnt;
  }
}

__global__ void k_cand_emit27(View v) {
  if (!v.dc[DC_REBUILD]) return;
  AGB_GRID_STRIDE(q, 27LL * v.natoms) {
    int n = v.nl_c27[q];
    if (n == 0) continue;
    int o = v.nl_o27[q];
    if (o + n > v.cap_cand) {
      set_err(v, AGB_ERR_CAND_CAP);
      continue;
    }
    int g = (int)(q / 27), c = (int)(q % 27);
    int I = v.inst_of[g];
    f4 a = v.pos[g];
    int m = 0;
    for_cell(v, I, v.atom_cell[3 * g] + c % 3 - 1, v.atom_cell[3 * g + 1] + (c / 3) % 3 - 1,
             v.atom_cell[3 * g + 2] + c / 9 - 1, [&](int j, const f4 &b) {
               if (j > g && cand_test(a, b, v.skin) && m < n) {
                 v.cand_j[o + m] = j;
                 v.cand_own[o + m] = g;
                 m++;
               }
             });
  }
}

/* per-atom candidate CSR and the build positions, only when rebuilding */
__global__ void k_cand_offsets(View v) {
  if (!v.dc[DC_REBUILD]) return;
  const int tot = v.dc[DC_CTOT];
  AGB_GRID_STRIDE(g, v.natoms) {
    int o = v.nl_o27[27 * g], e = (g + 1 < v.natoms) ? v.nl_o27[27 * (g + 1)] : tot;
    v.cand_off[g] = o;
    v.cand_cnt[g] = e - o;
    v.pos_ref[g] = v.pos[g];
    /* an overflowing build leaves no candidates (the evaluation is redone
       with larger buffers) */
    if (g == 0) v.dc[DC_NCAND] = tot <= v.cap_cand ? tot : 0;
  }
}

/* the reference's test on every candidate at the current positions */
__global__ void k_cand_flag(View v) {
  int n = min(v.dc[DC_NCAND], v.cap_cand);
  AGB_GRID_STRIDE(e, n) {
    float d2;
    v.cand_flag[e] = near_test(v.pos[v.cand_own[e]], v.pos[v.cand_j[e]], d2) ? 1 : 0;
  }
}

__global__ void k_cand_nl_emit(View v) {
  int n = min(v.dc[DC_NCAND], v.cap_cand);
  AGB_GRID_STRIDE(e, n) {
    if (!v.cand_flag[e]) continue;
    int o = v.cand_scan[e];
    if (o >= v.cap_nl) {
      set_err(v, AGB_ERR_NL_CAP);
      continue;
    }
    int g = v.cand_own[e], j = v.cand_j[e];
    float d2;
    near_test(v.pos[g], v.pos[j], d2);
    v.nl_tmp[o] = j;
    v.nl_d2[o] = d2;
    v.nl_own[o] = g;
  }
}

/* per-atom CSR of the filtered list: the scan at the atom's first and
   past-last candidate */
__global__ void k_cand_nl_offsets(View v) {
  const int n = min(v.dc[DC_NCAND], v.cap_cand), tot = v.dc[DC_NL];
  AGB_GRID_STRIDE(g, v.natoms) {
    int a = v.cand_off[g], b = a + v.cand_cnt[g];
    int sa = a < n ? v.cand_scan[a] : tot, sb = b < n ? v.cand_scan[b] : tot;
    v.nl_off[g] = sa;
    v.nl_count[g] = sb - sa;
  }
}

/* each atom's list in (float d^2, index) order (agbnp3.c:3766-3792,
   4062-4066): one thread per entry places it at its rank */
__global__ void k_nl_rank(View v) {
  int n = min(v.dc[DC_NL], v.cap_nl);
  AGB_GRID_STRIDE(e, n) {
    if (v.dc[DC_ERR] & AGB_ERR_NL_CAP) continue;
    int g = v.nl_own[e];
    int o = v.nl_off[g], m = v.nl_count[g];
    float d2 = v.nl_d2[e];
    int j = v.nl_tmp[e], rank = 0;
    for (int b = o; b < o + m; b++) {
      float db = v.nl_d2[b];
      rank += (db < d2) || (db == d2 && v.nl_tmp[b] < j);
    }
    v.nl_list[o + rank] = j;
  }
}

/* ------------------------------------------------------------------------ */
/* volumes: the overlap tree                                                */
/* ------------------------------------------------------------------------ */
template <typename R>
__device__ __forceinline__ R atom_alpha(const View &v, int g) {
  return pa<R>(v, PA_ALPHA)[g];
}
template <typename R>
__device__ __forceinline__ R atom_rinv(const View &v, int g) {
  return pa<R>(v, PA_RINV)[g];
}

template <typename R>
__device__ __forceinline__ Ov<R> atom_pair(const View &v, int i, int j) {
  return ogauss<R>(atom_alpha<R>(v, i), R(C_PFC), px<R>(v, i), py<R>(v, i), pz<R>(v, i), atom_alpha<R>(v, j),
                   R(C_PFC), px<R>(v, j), py<R>(v, j), pz<R>(v, j));
}

template <typename R>
struct Vec4;
template <>
struct Vec4<float> {
  static __device__ __forceinline__ void st(float *p, float a, float b, float c, float d) {
    *(float4 *)p = make_float4(a, b, c, d);
  }
  static __device__ __forceinline__ void ld(const float *p, float &a, float &b, float &c, float &d) {
    float4 t = *(const float4 *)p;
    a = t.x;
    b = t.y;
    c = t.z;
    d = t.w;
  }
};
template <>
struct Vec4<double> {
  static __device__ __forceinline__ void st(double *p, double a, double b, double c, double d) {
    ((double2 *)p)[0] = make_double2(a, b);
    ((double2 *)p)[1] = make_double2(c, d);
  }
  static __device__ __forceinline__ void ld(const double *p, double &a, double &b, double &c, double &d) {
    double2 t0 = ((const double2 *)p)[0], t1 = ((const double2 *)p)[1];
    a = t0.x;
    b = t0.y;
    c = t1.x;
    d = t1.y;
  }
};

template <typename R>
__device__ __forceinline__ void rec_put(const View &v, int m, int q, const Ov<R> &o) {
  R *b = (R *)v.rec[m] + (size_t)q * F_NUM;
  Vec4<R>::st(b, o.a, o.p, o.cx, o.cy);
  Vec4<R>::st(b + 4, o.cz, o.gvol, o.fp, o.fpp);
}

template <typename R>
__device__ __forceinline__ Ov<R> rec_load(const View &v, int m, int q) {
  const R *b = (const R *)v.rec[m] + (size_t)q * F_NUM;
  Ov<R> o;
  Vec4<R>::ld(b, o.a, o.p, o.cx, o.cy);
  Vec4<R>::ld(b + 4, o.cz, o.gvol, o.fp, o.fpp);
  o.gvolp = R(0); /* not stored */
  return o;
}

/* self-volume and surface-area contributions of one kept overlap of order
   M to its parent k (agbnp3_cpu_simd_kernels.c:1322-1345) */
template <typename R, int M>
__device__ __forceinline__ void vol_terms(const View &v, int k, const Ov<R> &o, double &dvol, double &dsurf) {
  const double coef = ((M & 1) ? 1.0 : -1.0) / M; /* (-1)^(M+1) / M */
  const R sgn = (M & 1) ? R(1) : R(-1);           /* M * coef */
  R h3 = sgn * o.fp * R(3) * f_rcp(o.a), h4 = R(0.5) * sgn * o.fp;
  R u1 = atom_alpha<R>(v, k) * o.gvol, u2 = R(-2) * u1;
  R v0 = u2 * (px<R>(v, k) - o.cx), v1 = u2 * (py<R>(v, k) - o.cy), v2 = u2 * (pz<R>(v, k) - o.cz);
  R d2 = v0 * v0 + v1 * v1 + v2 * v2;
  dvol = coef * (double)o.gvolp;
  dsurf = (double)((h3 * u1 + h4 * d2 * f_rcp(u1)) * atom_rinv<R>(v, k));
}

/* order 2: candidates are the near-list pairs, one thread per entry; the
   kept flags are scanned in list order, so the records of an atom stay
   contiguous and in its near-list order */
template <typename R>
__global__ void k_l2_count(View v) {
  /* after an overflow the list is incomplete: zero counts (the scan that
     follows reads them, and the evaluation is redone with larger buffers) */
  const bool skip = v.dc[DC_ERR] & (AGB_ERR_NL_CAP | AGB_ERR_TREE_CAP);
  const int n = min(v.dc[DC_NL], v.cap_nl);
  AGB_GRID_STRIDE(e, n) {
    if (skip) {
      v.lv_cnt[2][e] = 0;
      continue;
    }
    Ov<R> ov = atom_pair<R>(v, v.nl_own[e], v.nl_list[e]);
    v.lv_cnt[2][e] = kept(ov.gvolp) ? 1 : 0;
  }
}

/* sum of a[0..1] over the run of consecutive lanes holding this lane's key;
   returns whether this lane ends its run */
__device__ __forceinline__ bool seg_scan2(double &a0, double &a1, int key) {
  const int lane = threadIdx.x & 31;
  int kp = __shfl_up_sync(0xffffffffu, key, 1);
  int kn = __shfl_down_sync(0xffffffffu, key, 1);
  unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || kp != key);
  int start = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
  for (int o = 1; o < 32; o <<= 1) {
    bool take = lane - o >= start;
    double t0 = __shfl_up_sync(0xffffffffu, a0, o), t1 = __shfl_up_sync(0xffffffffu, a1, o);
    if (take) {
      a0 += t0;
      a1 += t1;
    }
  }
  return lane == 31 || kn != key;
}

/* warp-uniform loop over the entries; the first parent (the list's atom) is
   shared by runs of consecutive entries and its sums are reduced in the
   warp before the atomics */
template <typename R>
__global__ void k_l2_emit(View v) {
  if (v.dc[DC_ERR] & (AGB_ERR_NL_CAP | AGB_ERR_TREE_CAP)) return;
  const int n = min(v.dc[DC_NL], v.cap_nl);
  const int c2 = v.cap[2], total = v.dc[DC_L0 + 2];
  const int lane = threadIdx.x & 31;
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long base = ((long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < n;
       base += nwarps * 32) {
    const int e = (int)base + lane;
    int g = -1 - lane;
    double dvg = 0.0, dsg = 0.0;
    if (e < n && v.lv_cnt[2][e]) {
      int q = v.lv_off[2][e];
      g = v.nl_own[e];
      int j = v.nl_list[e];
      if (q < c2) {
        int se = v.nl_off[g] + v.nl_count[g]; /* end of g's list */
        int qend = se < n ? v.lv_off[2][se] : total;
        Ov<R> ov = atom_pair<R>(v, g, j);
        v.par[2][q] = g;
        v.par[2][c2 + q] = j;
        rec_put<R>(v, 2, q, ov);
        v.gend[2][q] = qend;
        double dv, ds;
        vol_terms<R, 2>(v, g, ov, dvg, dsg);
        vol_terms<R, 2>(v, j, ov, dv, ds);
        atomicAdd(&v.volumep[j], dv);
        atomicAdd(&v.surf[j], ds);
      } else {
        set_err(v, AGB_ERR_TREE_CAP);
        g = -1 - lane;
      }
    }
    if (seg_scan2(dvg, dsg, g) && g >= 0) {
      atomicAdd(&v.volumep[g], dvg);
      atomicAdd(&v.surf[g], dsg);
    }
  }
}

/* order M >= 3: overlap a combines with the last atom of every later
   overlap b of its group (same generating overlap one order down).  The
   count pass also records which siblings were kept (bit b - a - 1 of a
   64-bit mask; 0 for groups wider than 64, whose kept siblings the emit
   pass finds again by search) */
template <typename R, int M>
__global__ void k_lm_count(View v) {
  /* after an overflow the level below is incomplete: zero counts, which
     the scan that places this level's records reads (the evaluation is
     redone with larger buffers) */
  const bool skip = v.dc[DC_ERR] & (AGB_ERR_NL_CAP | AGB_ERR_TREE_CAP);
  const int n = min(v.dc[DC_L0 + M - 1], v.cap[M - 1]);
  const int cm = v.cap[M - 1];
  AGB_GRID_STRIDE(a, n) {
    if (skip) {
      v.lv_cnt[M][a] = 0;
      v.lv_mask[M][a] = 0ull;
      continue;
    }
    int ge = v.gend[M - 1][a], cnt = 0;
    unsigned long long mask = 0ull;
    const Ov<R> oa = rec_load<R>(v, M - 1, a);
    for (int b = a + 1; b < ge; b++) {
      int j = v.par[M - 1][(size_t)(M - 2) * cm + b];
      Ov<R> ov = ogauss<R>(oa.a, oa.p, oa.cx, oa.cy, oa.cz, atom_alpha<R>(v, j), R(C_PFC), px<R>(v, j), py<R>(v, j),
                           pz<R>(v, j));
      if (kept(ov.gvolp)) {
        cnt++;
        if (b - a <= 64) mask |= 1ull << (b - a - 1);
      }
    }
    v.lv_cnt[M][a] = cnt;
    v.lv_mask[M][a] = ge - a - 1 <= 64 ? mask : 0ull;
  }
}

/* sum of a[0..NN) over the run of consecutive lanes holding this lane's
   key; returns whether this lane ends its run */
template <typename T, int NN>
__device__ __forceinline__ bool seg_scan_n(T (&a)[NN], int key) {
  const int lane = threadIdx.x & 31;
  int kp = __shfl_up_sync(0xffffffffu, key, 1);
  int kn = __shfl_down_sync(0xffffffffu, key, 1);
  unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || kp != key);
  int start = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
  const int span = __reduce_max_sync(0xffffffffu, lane - start);
  for (int o = 1; o <= span; o <<= 1) {
    bool take = lane - o >= start;
#pragma unroll
    for (int c = 0; c < NN; c++) {
      T t = __shfl_up_sync(0xffffffffu, a[c], o);
      if (take) a[c] += t;
    }
  }
  return lane == 31 || kn != key;
}

/* one thread per order-M record q: its generating overlap a, its rank k
   among a's kept children, the k-th kept sibling b (from the mask, or by
   search), the record itself and its volume terms; the terms of the
   generator's parents are summed over the warp's run of records sharing
   the generator before the atomics */
template <typename R, int M>
__global__ void k_lm_emit(View v) {
  if (v.dc[DC_ERR] & (AGB_ERR_NL_CAP | AGB_ERR_TREE_CAP)) return;
  if (v.dc[DC_L0 + M] > v.cap[M]) { /* the records up to the capacity are still made, then redone */
    if (blockIdx.x == 0 && threadIdx.x == 0) set_err(v, AGB_ERR_TREE_CAP);
  }
  const int n = min(v.dc[DC_L0 + M], v.cap[M]);
  const int cm = v.cap[M - 1], cn = v.cap[M];
  const int lane = threadIdx.x & 31;
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long base = ((long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < n;
       base += nwarps * 32) {
    const int q = (int)base + lane;
    int a = -1 - lane;
    double sums[2 * (M - 1)];
#pragma unroll
    for (int k = 0; k < 2 * (M - 1); k++) sums[k] = 0.0;
    if (q < n) {
      a = v.lv_own[M][q];
      const int q0 = v.lv_off[M][a], rank = q - q0, qend = q0 + v.lv_cnt[M][a];
      const unsigned long long mask = v.lv_mask[M][a];
      const Ov<R> oa = rec_load<R>(v, M - 1, a);
      int j = 0;
      Ov<R> ov;
      if (mask) {
        unsigned long long mm = mask;
        for (int t = 0; t < rank; t++) mm &= mm - 1; /* drop the lower kept siblings */
        const int b = a + __ffsll((long long)mm);
        j = v.par[M - 1][(size_t)(M - 2) * cm + b];
        ov = ogauss<R>(oa.a, oa.p, oa.cx, oa.cy, oa.cz, atom_alpha<R>(v, j), R(C_PFC), px<R>(v, j), py<R>(v, j),
                       pz<R>(v, j));
      } else {
        const int ge = v.gend[M - 1][a];
        int c = -1;
        for (int b = a + 1; b < ge && c < rank; b++) {
          j = v.par[M - 1][(size_t)(M - 2) * cm + b];
          ov = ogauss<R>(oa.a, oa.p, oa.cx, oa.cy, oa.cz, atom_alpha<R>(v, j), R(C_PFC), px<R>(v, j), py<R>(v, j),
                         pz<R>(v, j));
          if (kept(ov.gvolp)) c++;
        }
      }
      double dv, ds;
#pragma unroll
      for (int k = 0; k < M - 1; k++) {
        const int pk = v.par[M - 1][(size_t)k * cm + a];
        v.par[M][(size_t)k * cn + q] = pk;
        vol_terms<R, M>(v, pk, ov, dv, ds);
        sums[2 * k] = dv;
        sums[2 * k + 1] = ds;
      }
      v.par[M][(size_t)(M - 1) * cn + q] = j;
      rec_put<R>(v, M, q, ov);
      v.gend[M][q] = qend;
      vol_terms<R, M>(v, j, ov, dv, ds);
      atomicAdd(&v.volumep[j], dv);
      atomicAdd(&v.surf[j], ds);
    }
    if (seg_scan_n(sums, a) && a >= 0) {
#pragma unroll
      for (int k = 0; k < M - 1; k++) {
        const int pk = v.par[M - 1][(size_t)k * cm + a];
        atomicAdd(&v.volumep[pk], sums[2 * k]);
        atomicAdd(&v.surf[pk], sums[2 * k + 1]);
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* scaling factors, filtered surface areas, cavity energy                   */
/* ------------------------------------------------------------------------ */
__global__ void k_scaling(View v) {
  AGB_GRID_STRIDE(g, v.natoms) {
    int I = v.inst_of[g];
    size_t N = v.natoms;
    if (g >= v.inst_begin[I] + v.inst_nheavy[I]) {
      v.sp[g] = 1.0;
      v.spe[g] = 0.0;
      v.surf_f[g] = v.psvol[g] = v.gammap[g] = 0.0;
      v.eatom[4 * N + g] = v.eatom[5 * N + g] = v.eatom[6 * N + g] = 0.0;
      continue;
    }
    double A = v.surf[g], f, fp;
    if (A < 0.0) { /* agbnp3.c:1104-1117 */
      f = fp = 0.0;
    } else {
      double t = A / (64.0 + A * A);
      f = A * t;
      fp = 2.0 * t * (1.0 - f);
    }
    double sf = A * f, r = v.r[g], vol = v.vols[g];
    v.surf_f[g] = sf;
    v.gammap[g] = (v.igamma[g] + v.sgamma[g]) * (f + A * fp);
    v.spe[g] = v.volumep[g] / vol;
    double q = (r - C_RINC) / r;
    double pr = r * (1.0 - q * q * q) / 3.0;
    v.psvol[g] = (fp * A + f) * pr;
    double vp = v.volumep[g] - sf * pr;
    v.volumep[g] = vp;
    v.sp[g] = vp / vol;
    v.eatom[4 * N + g] = v.igamma[g] * sf;
    v.eatom[5 * N + g] = v.sgamma[g] * sf;
    v.eatom[6 * N + g] = vp;
  }
}

/* exp(-d^2 / (4 Bi Bj)) as exp2 of a pre-scaled argument in float */
template <typename R>
struct GbExp;
template <>
struct GbExp<float> {
  static __device__ __forceinline__ float scale() { return -0.25f * 1.4426950408889634f; }
  static __device__ __forceinline__ float ex(float a) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(a));
    return y;
  }
};
template <>
struct GbExp<double> {
  static __device__ __forceinline__ double scale() { return -0.25; }
  static __device__ __forceinline__ double ex(double a) { return exp(a); }
};

/* cubic spline of one Q4 table at xh = a / h in [0, AGB_NA-1)
   (agbnp3_utils.c:229-252), divided by the descreening atom's radius R
   (the same for every atom of its radius type), stored per interval k as
   the cubic in t = xh - k, Q4/R = c0 + t (c1 + t (c2 + t c3)), one 16-byte
   (float) or 32-byte (double) record per lookup.  The spline's second
   derivatives at the interval ends are y2_k = 2 c2 / h^2 and
   y2_k+1 = (6 c3 + 2 c2) / h^2 (times 1/R), so the record also gives the
   derivative in t:
     exact:      c1 + 2 c2 t + 3 c3 t^2
     reference:  the exact one minus (3 t^2 - 1) h^2 y2_k+1 / 3
                 (agbnp3_utils.c:247-249 adds the y2_k+1 curvature term
                 where the spline derivative subtracts it)
   i.e. c1 + 2 c3 + 2 c2 / 3 + 2 c2 t - (3 c3 + 2 c2) t^2, and
   d(Q4/R)/da = (derivative in t) / h. */
template <typename R>
struct Tab;
template <>
struct Tab<float> {
  typedef float4 T;
  static __device__ __forceinline__ float4 ld(const float4 *p) { return __ldg(p); }
  static __device__ __forceinline__ const float4 *val(const View &v) { return v.tabv_f; }
};
template <>
struct Tab<double> {
  typedef double4 T;
  static __device__ __forceinline__ double4 ld(const double4 *p) {
    const double2 *q = (const double2 *)p;
    double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
  }
  static __device__ __forceinline__ const double4 *val(const View &v) { return v.tabv_d; }
};

/* the same with the interval index clamped to AGB_NA-1, whose record is all
   zeros: beyond the table (a >= 20) the value and the derivative are 0
   without a test */
template <typename R>
__device__ __forceinline__ R spline_z(const typename Tab<R>::T *tv, int slot, R xh) {
  int k = min((int)xh, AGB_NA - 1);
  R t = xh - R(k);
  typename Tab<R>::T c = Tab<R>::ld(tv + (size_t)slot * AGB_NA + k);
  return c.x + t * (c.y + t * (c.z + t * c.w));
}

/* value and derivative in t; REF: the reference's derivative, else exact.
   The interval index is clamped to AGB_NA-1 (an all-zero record), so
   beyond the table both are 0. */
template <typename R, bool REF>
__device__ __forceinline__ R spline_d(const typename Tab<R>::T *tv, int slot, R xh, R &fph) {
  int k = min((int)xh, AGB_NA - 1);
  R t = xh - R(k);
  typename Tab<R>::T c = Tab<R>::ld(tv + (size_t)slot * AGB_NA + k);
  R d0 = REF ? c.y + R(2) * c.w + R(2.0 / 3.0) * c.z : c.y;
  R d2 = REF ? -(R(3) * c.w + R(2) * c.z) : R(3) * c.w;
  fph = d0 + t * (R(2) * c.z + t * d2);
  return c.x + t * (c.y + t * (c.z + t * c.w));
}

template <typename R>
__global__ void k_pack_geom(View v) {
  AGB_GRID_STRIDE(g, v.natoms) {
    R ri = R(1) / (R)v.r[g];
    const int s = v.atom_slot[g];
    pa<R>(v, PA_X)[s] = px<R>(v, (int)g);
    pa<R>(v, PA_Y)[s] = py<R>(v, (int)g);
    pa<R>(v, PA_Z)[s] = pz<R>(v, (int)g);
    pa<R>(v, PA_RINV)[g] = ri;
    pa<R>(v, PA_RH)[s] = ri * R((AGB_NA - 1) / C_AMAX);
    pa<R>(v, PA_ALPHA)[g] = R(C_KFC) / ((R)v.r[g] * (R)v.r[g]);
    pa<R>(v, PA_Q)[s] = (R)v.charge[g];
    v.slot_type[s] = v.rtype[g];
    v.slot_hvcol[s] = v.hvslot[v.rtype[g]] * AGB_NA;
    v.acc_beta[g] = 0.0;
  }
}

template <typename R>
__global__ void k_pack_sp(View v) {
  AGB_GRID_STRIDE(g, v.natoms) {
    R sp = (R)v.sp[g];
    pa<R>(v, PA_SP)[v.atom_slot[g]] = sp;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) v.dc[DC_DESQ] = 0;
}

/* partner range of a work item: chunk w.w of nch of [p0, p1) */
/* partner range [c0, c1) of an item's chunk: the item's code holds its
   chunk index c and its instance's chunk count n as c + 64 n */
__device__ __forceinline__ void chunk_range(int p0, int p1, int code, int &c0, int &c1) {
  const int c = code & 63, nch = code >> 6;
  long long len = p1 - p0;
  c0 = p0 + (int)(len * c / nch);
  c1 = p0 + (int)(len * (c + 1) / nch);
}

/* ------------------------------------------------------------------------ */
/* invb: descreening sums (agbnp3_cpu_simd_kernels.c:500-678).  Each block  */
/* owns up to ITILE atoms of one instance and one chunk of its heavy        */
/* descreeners, staged through shared memory; per-tile sums in R are added  */
/* to a double accumulator.                                                 */
/* ------------------------------------------------------------------------ */
#define ITILE 128

/* a staged partner: position and 1/(R h) in one vector record, the
   descreening weight and the offset of its radius type's column of tables
   (type * AGB_NA records) in another */
template <typename R>
struct alignas(4 * sizeof(R)) Part4 {
  R x, y, z, rh;
};
template <typename R>
struct alignas(2 * sizeof(R)) PartW {
  R w;
  int t;
};

/* one staged group of partners against a thread's two atoms; SELF: the
   group may hold the atoms themselves (skipped) */
template <typename R, bool SELF>
__device__ __forceinline__ void desc_group(const Part4<R> *sp4, const PartW<R> *spw, int t0, int t1, int j0,
                                           const int (&g)[2], const R (&xg)[2], const R (&yg)[2], const R (&zg)[2],
                                           const typename Tab<R>::T *const (&rowp)[2], R (&part)[2]) {
#pragma unroll 4
  for (int t = t0; t < t1; t++) {
    Part4<R> a = sp4[t];
    PartW<R> b = spw[t];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      R dx = a.x - xg[u], dy = a.y - yg[u], dz = a.z - zg[u];
      R xh = p_sqrt(dx * dx + dy * dy + dz * dz) * a.rh;
      if (xh < R(AGB_NA - 1) && (!SELF || j0 + t != g[u])) {
        const int k = (int)xh;
        R tt = xh - R(k);
        typename Tab<R>::T c = Tab<R>::ld(rowp[u] + b.t + k);
        part[u] += b.w * (c.x + tt * (c.y + tt * (c.z + tt * c.w)));
      }
    }
  }
}

/* float bounds that contain a working-precision value */
__device__ __forceinline__ float lo_f(float x) { return x; }
__device__ __forceinline__ float hi_f(float x) { return x; }
__device__ __forceinline__ float lo_f(double x) { return __double2float_rd(x); }
__device__ __forceinline__ float hi_f(double x) { return __double2float_ru(x); }

__device__ __forceinline__ void warp_minmax(float &lo, float &hi) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
}

/* bounding box and smallest 1/(hR) of every 32-slot tile of the pair slots
   (one warp per tile), for the range culling of the descreening pass */
template <typename R>
__global__ void k_tile_box(View v) {
  const R *X = pa<R>(v, PA_X), *Y = pa<R>(v, PA_Y), *Z = pa<R>(v, PA_Z), *RH = pa<R>(v, PA_RH);
  const int lane = threadIdx.x & 31;
  const long long ntile = ((long long)v.natoms + 31) / 32;
  for (long long T = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; T < ntile;
       T += ((long long)gridDim.x * blockDim.x) >> 5) {
    const long long s = T * 32 + lane;
    const bool a = s < v.natoms;
    float lx = a ? lo_f(X[s]) : INFINITY, hx = a ? hi_f(X[s]) : -INFINITY;
    float ly = a ? lo_f(Y[s]) : INFINITY, hy = a ? hi_f(Y[s]) : -INFINITY;
    float lz = a ? lo_f(Z[s]) : INFINITY, hz = a ? hi_f(Z[s]) : -INFINITY;
    float rh = a ? lo_f(RH[s]) : INFINITY, unused = -INFINITY;
    warp_minmax(lx, hx);
    warp_minmax(ly, hy);
    warp_minmax(lz, hz);
    warp_minmax(rh, unused);
    if (lane == 0) {
      v.tbox[2 * T] = make_float4(lx, ly, lz, rh);
      v.tbox[2 * T + 1] = make_float4(hx, hy, hz, 0.f);
    }
  }
}

/* whether any atom of the box [ilo, ihi] can lie within the Q4 tables'
   range (a < 20) of a descreener of tile T: the boxes' distance D against
   20 h R = (AGB_NA - 1) / (1/(hR)), with a 0.1 % margin that covers the
   rounding of the pair pass's own distance (so every pair of a culled tile
   would fail the pass's range test, and culling changes no bit) */
__device__ __forceinline__ bool tile_in_range(const float4 *tbox, long long T, float4 ilo, float4 ihi) {
  const float4 lo = tbox[2 * T], hi = tbox[2 * T + 1];
  const float dx = fmaxf(0.f, fmaxf(lo.x - ihi.x, ilo.x - hi.x));
  const float dy = fmaxf(0.f, fmaxf(lo.y - ihi.y, ilo.y - hi.y));
  const float dz = fmaxf(0.f, fmaxf(lo.z - ihi.z, ilo.z - hi.z));
  const float lim = float(AGB_NA - 1) * 1.001f / lo.w;
  return dx * dx + dy * dy + dz * dz < lim * lim;
}

/* blocks of ITILE/2 threads; warp w holds atoms [64 w, 64 w + 64) of the
   ITILE-atom item, two per lane.  Per staged group of partners each warp
   tests the group's (at most five) 32-slot partner tiles against the
   bounding box of its own atoms and skips the tiles beyond the Q4 range
   (their every term is exactly 0); a group no warp needs is not staged.
   FP32: sixteen resident blocks per SM (64 registers), measured faster
   than the compiler's own choice of 40 registers with spills at 25,000 and
   100,000 atoms and in the 512-instance batch; FP64: eight. */
template <typename R>
struct DescBlocks {
  static constexpr int v = sizeof(R) == 4 ? 16 : 8;
};
template <typename R>
__global__ void __launch_bounds__(ITILE / 2, DescBlocks<R>::v) k_descreen_t(View v, const int4 *__restrict__ items, int nitems,
                                                          int nch) {
  AGB_SHARED Part4<R> sp4[ITILE];
  AGB_SHARED PartW<R> spw[ITILE];
  AGB_SHARED float4 sbox[ITILE / 64][2];
  const R *X = pa<R>(v, PA_X), *Y = pa<R>(v, PA_Y), *Z = pa<R>(v, PA_Z);
  const R *RH = pa<R>(v, PA_RH), *W = pa<R>(v, PA_SP); /* the tables carry 1/R of the descreener */
  const typename Tab<R>::T *tab = Tab<R>::val(v);
  const int nt = v.ntypes;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    int4 w = items[it];
    int g[2];
    bool act[2];
    R xg[2], yg[2], zg[2];
    int row[2];
    const typename Tab<R>::T *rowp[2];
    double acc[2] = {0.0, 0.0};
#pragma unroll
    for (int u = 0; u < 2; u++) {
      g[u] = w.y + 64 * wid + lane + 32 * u;
      act[u] = g[u] < w.z;
      xg[u] = act[u] ? X[g[u]] : R(0);
      yg[u] = act[u] ? Y[g[u]] : R(0);
      zg[u] = act[u] ? Z[g[u]] : R(0);
      row[u] = act[u] ? v.slot_type[g[u]] * nt : 0;
      rowp[u] = tab + (size_t)row[u] * AGB_NA;
    }
    {
      /* this warp's bounding box (empty when it holds no atom) */
      float lx = INFINITY, ly = INFINITY, lz = INFINITY, hx = -INFINITY, hy = -INFINITY, hz = -INFINITY;
#pragma unroll
      for (int u = 0; u < 2; u++)
        if (act[u]) {
          lx = fminf(lx, lo_f(xg[u]));
          ly = fminf(ly, lo_f(yg[u]));
          lz = fminf(lz, lo_f(zg[u]));
          hx = fmaxf(hx, hi_f(xg[u]));
          hy = fmaxf(hy, hi_f(yg[u]));
          hz = fmaxf(hz, hi_f(zg[u]));
        }
      warp_minmax(lx, hx);
      warp_minmax(ly, hy);
      warp_minmax(lz, hz);
      __syncwarp(); /* the previous item's readers of this warp's box are done */
      if (lane == 0) {
        sbox[wid][0] = make_float4(lx, ly, lz, 0.f);
        sbox[wid][1] = make_float4(hx, hy, hz, 0.f);
      }
      __syncwarp();
    }
    int p0 = v.inst_begin[w.x], c0, c1;
    chunk_range(p0, p0 + v.inst_nheavy[w.x], w.w, c0, c1);
    for (int j0 = c0; j0 < c1; j0 += ITILE) {
      int n = min(ITILE, c1 - j0);
      const int T0 = j0 >> 5, ntl = ((j0 + n - 1) >> 5) - T0 + 1; /* ntl <= 5 */
      bool f = false;
      if (lane < ntl) f = tile_in_range(v.tbox, T0 + lane, sbox[wid][0], sbox[wid][1]);
      const unsigned mask = __ballot_sync(0xffffffffu, f);
      /* also the barrier after the previous group's readers of sp4/spw */
      if (!__syncthreads_or(mask != 0u)) continue;
      AGB_COOP_FOR(t, n) {
        Part4<R> a;
        a.x = X[j0 + t];
        a.y = Y[j0 + t];
        a.z = Z[j0 + t];
        a.rh = RH[j0 + t];
        sp4[t] = a;
        PartW<R> b;
        b.w = W[j0 + t];
        b.t = v.slot_type[j0 + t] * AGB_NA;
        spw[t] = b;
      }
      AGB_SYNC();
      if (act[0] && mask) {
        R part[2] = {R(0), R(0)};
        /* the item's own atoms are among the partners only when the staged
           range overlaps the item (warp-uniform) */
        const bool self = j0 < w.z && j0 + n > w.y;
        if (mask == (1u << ntl) - 1u) { /* every tile in range */
          if (self)
            desc_group<R, true>(sp4, spw, 0, n, j0, g, xg, yg, zg, rowp, part);
          else
            desc_group<R, false>(sp4, spw, 0, n, j0, g, xg, yg, zg, rowp, part);
        } else {
          for (int k = 0; k < ntl; k++)
            if ((mask >> k) & 1u) {
              const int t0 = max(0, (T0 + k) * 32 - j0), t1 = min(n, (T0 + k + 1) * 32 - j0);
              if (self)
                desc_group<R, true>(sp4, spw, t0, t1, j0, g, xg, yg, zg, rowp, part);
              else
                desc_group<R, false>(sp4, spw, t0, t1, j0, g, xg, yg, zg, rowp, part);
            }
        }
        acc[0] += (double)part[0];
        acc[1] += (double)part[1];
      }
    }
#pragma unroll
    for (int u = 0; u < 2; u++)
      if (act[u]) atomicAdd(&v.acc_beta[v.slot_atom[g[u]]], acc[u]);
  }
}

/* FP32 descreening with the heavy-descreener tables (View::tabh_f) in
   shared memory: one block of DS_WARPS warps per SM.  Each warp takes half
   an item (64 of its ITILE atoms, two per lane) from a device counter,
   tests 32 partner tiles at a time against its atoms' bounding box (one
   tile per lane) and stages each 32-slot tile in range itself, so after
   the tables' copy no block barrier is needed. */
#define DS_WARPS 32
#define DS_GROUP 32 /* partners staged per warp: one 32-slot tile */

/* the work unit of the c-th take from a device counter, for U units: the
   takes run down the columns of a 148-row table of the units in order, so
   that the warps of one SM, taking in a burst, get units far apart in the
   list (neighbouring units cover neighbouring atoms and cost alike);
   returns -1 for a take beyond the table and U + 1 for an empty cell */
__device__ __forceinline__ int take_unit(int c, int U) {
  const int K = (U + 147) / 148;
  if (c >= 148 * K) return -1;
  const int u = (c % 148) * K + c / 148;
  return u < U ? u : U + 1;
}
template <bool SELF>
__device__ __forceinline__ void desc_group_s(const Part4<float> *sp4, const PartW<float> *spw, int t0, int t1, int j0,
                                             const int (&g)[2], const float (&xg)[2], const float (&yg)[2],
                                             const float (&zg)[2], const float4 *ts, const int (&ro)[2],
                                             float (&part)[2]) {
#pragma unroll 4
  for (int t = t0; t < t1; t++) {
    const Part4<float> a = sp4[t];
    const PartW<float> b = spw[t];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const float dx = a.x - xg[u], dy = a.y - yg[u], dz = a.z - zg[u];
      const float xh = p_sqrt(dx * dx + dy * dy + dz * dz) * a.rh;
      if (xh < float(AGB_NA - 1) && (!SELF || j0 + t != g[u])) {
        const int k = (int)xh;
        const float tt = xh - float(k);
        const float4 c = ts[ro[u] + b.t + k];
        part[u] += b.w * (c.x + tt * (c.y + tt * (c.z + tt * c.w)));
      }
    }
  }
}

__global__ void __launch_bounds__(DS_WARPS * 32, 1) k_descreen_s(View v, const int4 *__restrict__ items, int nitems) {
  extern __shared__ float4 ds_dyn[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  Part4<float> *sp4 = reinterpret_cast<Part4<float> *>(ds_dyn) + wid * DS_GROUP;
  PartW<float> *spw = reinterpret_cast<PartW<float> *>(ds_dyn + DS_WARPS * DS_GROUP) + wid * DS_GROUP;
  float4 *ts = ds_dyn + DS_WARPS * DS_GROUP + DS_WARPS * DS_GROUP / 2;
  {
    const int nrec = v.ntypes * v.nhv * AGB_NA;
    for (int q = threadIdx.x; q < nrec; q += blockDim.x) ts[q] = __ldg(v.tabh_f + q);
    __syncthreads();
  }
  const float *X = pa<float>(v, PA_X), *Y = pa<float>(v, PA_Y), *Z = pa<float>(v, PA_Z);
  const float *RH = pa<float>(v, PA_RH), *W = pa<float>(v, PA_SP); /* the tables carry 1/R of the descreener */
  const int nhv = v.nhv;
  const int U = 2 * nitems;
  int u = 0;
  if (lane == 0) u = take_unit(atomicAdd(&v.dc[DC_DESQ], 1), U);
  u = __shfl_sync(FULLMASK, u, 0);
  while (u >= 0) {
    if (u < U) {
      const int4 w = items[u >> 1];
      int g[2], ro[2];
      bool act[2];
      float xg[2], yg[2], zg[2];
#pragma unroll
      for (int k = 0; k < 2; k++) {
        g[k] = w.y + 64 * (u & 1) + lane + 32 * k;
        act[k] = g[k] < w.z;
        xg[k] = act[k] ? X[g[k]] : 0.f;
        yg[k] = act[k] ? Y[g[k]] : 0.f;
        zg[k] = act[k] ? Z[g[k]] : 0.f;
        ro[k] = (act[k] ? v.slot_type[g[k]] * nhv : 0) * AGB_NA; /* the row of the atom's radius type */
      }
      if (__any_sync(FULLMASK, act[0])) {
        /* this warp's bounding box */
        float lx = INFINITY, ly = INFINITY, lz = INFINITY, hx = -INFINITY, hy = -INFINITY, hz = -INFINITY;
#pragma unroll
        for (int k = 0; k < 2; k++)
          if (act[k]) {
            lx = fminf(lx, xg[k]);
            ly = fminf(ly, yg[k]);
            lz = fminf(lz, zg[k]);
            hx = fmaxf(hx, xg[k]);
            hy = fmaxf(hy, yg[k]);
            hz = fmaxf(hz, zg[k]);
          }
        warp_minmax(lx, hx);
        warp_minmax(ly, hy);
        warp_minmax(lz, hz);
        const float4 blo = make_float4(lx, ly, lz, 0.f), bhi = make_float4(hx, hy, hz, 0.f);
        double acc[2] = {0.0, 0.0};
        int p0 = v.inst_begin[w.x], c0, c1;
        chunk_range(p0, p0 + v.inst_nheavy[w.x], w.w, c0, c1);
        /* the chunk's 32-slot partner tiles, 32 tiles tested at once (one
           per lane), then each tile in range staged and summed */
        const int Tb = c0 >> 5, Te = (c1 - 1) >> 5;
        for (int W0 = Tb; c1 > c0 && W0 <= Te; W0 += 32) {
          const int T = W0 + lane;
          unsigned mask = __ballot_sync(FULLMASK, T <= Te && tile_in_range(v.tbox, T, blo, bhi));
          /* the tiles in range, the next one's partner loaded into registers
             while the current one is summed */
          int T1 = W0 + __ffs(mask) - 1, t0 = 0, n = 0;
          Part4<float> a;
          PartW<float> b;
          const auto fetch = [&](int Tn) {
            t0 = max(c0, 32 * Tn);
            n = min(c1, 32 * Tn + 32) - t0;
            if (lane < n) {
              const int j = t0 + lane;
              a.x = X[j];
              a.y = Y[j];
              a.z = Z[j];
              a.rh = RH[j];
              b.w = W[j];
              b.t = v.slot_hvcol[j];
            }
          };
          if (mask) fetch(T1);
          while (mask) {
            mask &= mask - 1;
            const int c0t = t0, nt0 = n;
            __syncwarp(); /* the previous tile's readers are done */
            if (lane < nt0) {
              sp4[lane] = a;
              spw[lane] = b;
            }
            __syncwarp();
            if (mask) fetch(W0 + __ffs(mask) - 1);
            if (act[0]) {
              float part[2] = {0.f, 0.f};
              if (c0t < w.z && c0t + nt0 > w.y) /* the item's own atoms among the partners */
                desc_group_s<true>(sp4, spw, 0, nt0, c0t, g, xg, yg, zg, ts, ro, part);
              else
                desc_group_s<false>(sp4, spw, 0, nt0, c0t, g, xg, yg, zg, ts, ro, part);
              acc[0] += (double)part[0];
              acc[1] += (double)part[1];
            }
          }
        }
#pragma unroll
        for (int k = 0; k < 2; k++)
          if (act[k]) atomicAdd(&v.acc_beta[v.slot_atom[g[k]]], acc[k]);
      }
    }
    if (lane == 0) u = take_unit(atomicAdd(&v.dc[DC_DESQ], 1), U);
    u = __shfl_sync(FULLMASK, u, 0);
  }
}

/* inverse Born radius, its filter, Born radius, vdW energy
   (agbnp3_cpu_simd_kernels.c:605, agbnp3.c:1174-1188, 1466-1487,
   agbnp3_utils.c:615-670) */
template <typename R>
__global__ void k_born(View v) {
  size_t N = v.natoms;
  AGB_GRID_STRIDE(g, v.natoms) {
    double beta = 1.0 / (v.r[g] - C_RINC) - v.acc_beta[g] / (4.0 * C_PI);
    double bf, bd;
    if (beta < 0.0) {
      bf = 0.02;
      bd = 0.0;
    } else {
      bf = sqrt(0.02 * 0.02 + beta * beta);
      bd = beta / bf;
    }
    double b = 1.0 / bf, t = b + C_RW;
    v.bfil[g] = bf;
    v.bder[g] = bd;
    v.br[g] = b;
    v.brw[g] = 3.0 * b * b / (t * t * t * t);
    double a3 = 1.0 / (t * t * t);
    v.eatom[2 * N + g] = v.ialpha[g] * a3;
    v.eatom[3 * N + g] = v.salpha[g] * a3;
    v.eatom[N + g] = 0.0;
    v.dera[g] = 0.0;
    pa<R>(v, PA_B)[v.atom_slot[g]] = (R)b;
    pa<R>(v, PA_BINV)[v.atom_slot[g]] = (R)bf;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) v.dc[DC_AGBQ] = 0;
}

/* ------------------------------------------------------------------------ */
/* agb: GB pair energy, gradient at constant Born radii and A_i             */
/* (agbnp3_cpu_simd_kernels.c:66-151, 329-460), all ordered pairs           */
/* ------------------------------------------------------------------------ */
template <typename R>
__global__ void __launch_bounds__(ITILE) k_agb_t(View v, const int4 *__restrict__ items, int nitems, int nch) {
  AGB_SHARED R sx[ITILE], sy[ITILE], sz[ITILE], sq[ITILE], sb[ITILE], sbi[ITILE];
  const R *X = pa<R>(v, PA_X), *Y = pa<R>(v, PA_Y), *Z = pa<R>(v, PA_Z);
  const R *Q = pa<R>(v, PA_Q), *Bv = pa<R>(v, PA_B), *BI = pa<R>(v, PA_BINV);
  size_t N = v.natoms;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    int4 w = items[it];
    int g = w.y + threadIdx.x;
    bool act = g < w.z;
    int c0, c1;
    chunk_range(v.inst_begin[w.x], v.inst_begin[w.x + 1], w.w, c0, c1);
    double df = v.inst_df[w.x];
    R xg = act ? X[g] : R(0), yg = act ? Y[g] : R(0), zg = act ? Z[g] : R(0);
    R bg = act ? Bv[g] : R(1), cg = act ? GbExp<R>::scale() * BI[g] : R(0);
    double e = 0, gx = 0, gy = 0, gz = 0, at = 0;
    for (int j0 = c0; j0 < c1; j0 += ITILE) {
      int n = min(ITILE, c1 - j0);
      AGB_SYNC();
      AGB_COOP_FOR(t, n) {
        sx[t] = X[j0 + t];
        sy[t] = Y[j0 + t];
        sz[t] = Z[j0 + t];
        sq[t] = Q[j0 + t];
        sb[t] = Bv[j0 + t];
        sbi[t] = BI[j0 + t];
      }
      AGB_SYNC();
      if (act) {
        R pe = 0, px_ = 0, py_ = 0, pz_ = 0, pat = 0;
        for (int t = 0; t < n; t++) {
          R dx = sx[t] - xg, dy = sy[t] - yg, dz = sz[t] - zg;
          R d2 = dx * dx + dy * dy + dz * dz;
          if (!(d2 > R(0))) continue; /* the atom itself and coincident atoms */
          R bb = bg * sb[t];
          R et = GbExp<R>::ex(cg * sbi[t] * d2);
          R f = p_rsqrt(d2 + bb * et);
          R qf3 = sq[t] * f * f * f;
          pe += sq[t] * f;
          R mw = (R(1) - R(0.25) * et) * qf3;
          px_ += mw * dx;
          py_ += mw * dy;
          pz_ += mw * dz;
          pat += (bb + R(0.25) * d2) * et * qf3;
        }
        e += (double)pe;
        gx += (double)px_;
        gy += (double)py_;
        gz += (double)pz_;
        at += (double)pat;
      }
    }
    if (act) {
      /* qj and the factor 2 df qi are applied once per atom */
      const int ga = v.slot_atom[g];
      double qi = v.charge[ga], w2 = 2.0 * df * qi;
      atomicAdd(&v.eatom[N + ga], C_TOKCAL * 0.5 * w2 * e);
      atomicAdd(&v.g_gb[3 * ga], w2 * gx);
      atomicAdd(&v.g_gb[3 * ga + 1], w2 * gy);
      atomicAdd(&v.g_gb[3 * ga + 2], w2 * gz);
      atomicAdd(&v.dera[ga], qi * at);
    }
  }
}

/* self energy, q2ab and abrw (agbnp3_cpu_simd_kernels.c:359, 444-449) */
template <typename R>
__global__ void k_agb_post(View v) {
  AGB_GRID_STRIDE(g, v.natoms) {
    double df = v.inst_df[v.inst_of[g]];
    double q = v.charge[g], b = v.br[g];
    v.eatom[g] = C_TOKCAL * df * q * q / b;
    double q2ab = (q * q + v.dera[g] * b) * v.bder[g];
    double abrw = (v.ialpha[g] + v.salpha[g]) * v.brw[g] * v.bder[g];
    v.q2ab[g] = q2ab;
    v.abrw[g] = abrw;
    pa<R>(v, PA_Q2AB)[v.atom_slot[g]] = (R)q2ab;
    pa<R>(v, PA_ABRW)[v.atom_slot[g]] = (R)abrw;
    v.deru[g] = v.derv[g] = 0.0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) v.dc[DC_GBDQ] = 0;
}

/* ------------------------------------------------------------------------ */
/* gbders: GB and vdW gradients through the Born radii at constant self      */
/* volumes and U_i, V_i (agbnp3_cpu_simd_kernels.c:681-904).  Thread a adds  */
/* for each partner b the pair force of both descreening directions; U_a,    */
/* V_a collect the atoms a descreens.                                        */
/* ------------------------------------------------------------------------ */
template <typename R>
__global__ void __launch_bounds__(ITILE) k_gbders_t(View v, const int4 *__restrict__ items, int nitems,
                                                    int nch) {
  AGB_SHARED R sx[ITILE], sy[ITILE], sz[ITILE], srh[ITILE], ssp[ITILE], sq2[ITILE], sab[ITILE];
  AGB_SHARED int st[ITILE];
  const R *X = pa<R>(v, PA_X), *Y = pa<R>(v, PA_Y), *Z = pa<R>(v, PA_Z);
  const R *RH = pa<R>(v, PA_RH), *SP = pa<R>(v, PA_SP);
  const R *Q2 = pa<R>(v, PA_Q2AB), *AB = pa<R>(v, PA_ABRW);
  const typename Tab<R>::T *tv = Tab<R>::val(v);
  const bool ref = v.compat != 0;
  const int nt = v.ntypes;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    int4 w = items[it];
    int g = w.y + threadIdx.x;
    bool act = g < w.z;
    int a0 = v.inst_begin[w.x], hh = a0 + v.inst_nheavy[w.x], a1 = v.inst_begin[w.x + 1];
    /* a tile of hydrogens only needs heavy partners */
    int c0, c1;
    chunk_range(a0, w.y >= hh ? hh : a1, w.w, c0, c1);
    bool heavy = g < hh;
    R xg = act ? X[g] : R(0), yg = act ? Y[g] : R(0), zg = act ? Z[g] : R(0);
    R rhg = act ? RH[g] : R(0), spg = act ? SP[g] : R(0);
    R q2g = act ? Q2[g] : R(0), abg = act ? AB[g] : R(0);
    int tg = act ? v.slot_type[g] : 0;
    double U = 0, V = 0, fx = 0, fy = 0, fz = 0, vx = 0, vy = 0, vz = 0;
    for (int j0 = c0; j0 < c1; j0 += ITILE) {
      int n = min(ITILE, c1 - j0);
      AGB_SYNC();
      AGB_COOP_FOR(t, n) {
        sx[t] = X[j0 + t];
        sy[t] = Y[j0 + t];
        sz[t] = Z[j0 + t];
        srh[t] = RH[j0 + t];
        ssp[t] = SP[j0 + t];
        sq2[t] = Q2[j0 + t];
        sab[t] = AB[j0 + t];
        st[t] = v.slot_type[j0 + t];
      }
      AGB_SYNC();
      if (act) {
        R pu = 0, pv = 0, pfx = 0, pfy = 0, pfz = 0, pvx = 0, pvy = 0, pvz = 0;
        int tend = heavy ? n : min(n, hh - j0); /* hydrogens: heavy partners only */
        for (int t = 0; t < tend; t++) {
          int b = j0 + t;
          R dx = sx[t] - xg, dy = sy[t] - yg, dz = sz[t] - zg;
          R d2 = dx * dx + dy * dy + dz * dz;
          if (!(d2 > R(0))) continue;
          R id = p_rsqrt(d2);
          R d = d2 * id;
          R ht = R(0), ut = R(0);
          if (heavy) { /* b descreened by a: table (type b, type a), radius of a */
            R xh = d * rhg;
            if (xh < R(AGB_NA - 1)) {
              R fp;
              R f = ref ? spline_d<R, true>(tv, st[t] * nt + tg, xh, fp) : spline_d<R, false>(tv, st[t] * nt + tg, xh, fp);
              R q = f, dq = fp * rhg;
              pu += sq2[t] * q;
              pv += sab[t] * q;
              ht += sq2[t] * dq * spg;
              ut += sab[t] * dq * spg;
            }
          }
          if (b < hh) { /* a descreened by b: table (type a, type b), radius of b */
            R xh = d * srh[t];
            if (xh < R(AGB_NA - 1)) {
              R fp;
              if (ref)
                spline_d<R, true>(tv, tg * nt + st[t], xh, fp);
              else
                spline_d<R, false>(tv, tg * nt + st[t], xh, fp);
              R dq = fp * srh[t] * ssp[t];
              ht += q2g * dq;
              ut += abg * dq;
            }
          }
          ht *= id;
          ut *= id;
          pfx += ht * dx;
          pfy += ht * dy;
          pfz += ht * dz;
          pvx += ut * dx;
          pvy += ut * dy;
          pvz += ut * dz;
        }
        U += (double)pu;
        V += (double)pv;
        fx += (double)pfx;
        fy += (double)pfy;
        fz += (double)pfz;
        vx += (double)pvx;
        vy += (double)pvy;
        vz += (double)pvz;
      }
    }
    if (act) {
      const double f4p = 1.0 / (4.0 * C_PI);
      double kg = f4p * v.inst_df[w.x];
      const int ga = v.slot_atom[g];
      atomicAdd(&v.g_gb[3 * ga], kg * fx);
      atomicAdd(&v.g_gb[3 * ga + 1], kg * fy);
      atomicAdd(&v.g_gb[3 * ga + 2], kg * fz);
      atomicAdd(&v.g_vw[3 * ga], f4p * vx);
      atomicAdd(&v.g_vw[3 * ga + 1], f4p * vy);
      atomicAdd(&v.g_vw[3 * ga + 2], f4p * vz);
      if (heavy) {
        atomicAdd(&v.deru[ga], U);
        atomicAdd(&v.derv[ga], V);
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* symmetric pair passes: each warp owns an i block of NI 32-atom tiles     */
/* (lane l keeps atoms I+l, I+32+l, ...) and walks a run of 32-atom j tiles  */
/* of the same instance starting at the block.  The j atoms' operands and    */
/* their partial sums rotate through the warp with __shfl_sync: in step r    */
/* lane l holds j atom J+((l+r) mod 32), evaluates its pairs with its NI i   */
/* atoms when i < j, and after 32 steps each j atom's sums are back in its   */
/* lane.  Every unordered pair is evaluated once, NI per lane and step.      */
/* Partial sums are in the working precision over a j tile (j side) or a    */
/* j run (i side), then double.                                              */
/* ------------------------------------------------------------------------ */

template <typename T>
__device__ __forceinline__ T rot1(T x) {
  return __shfl_sync(FULLMASK, x, (threadIdx.x + 1) & 31);
}

/* agb: GB pair energy, constant-B gradient, A_i (agbnp3_cpu_simd_kernels.c:
   66-151, 329-460).  A lane keeps AGB_NI i atoms (I+l, I+32+l, ...), so
   each rotation step evaluates AGB_NI pairs with one set of shuffles.
   Interior j tiles (all valid, after the i block) skip the per-pair index
   tests. */
/* i atoms per lane of the symmetric passes: in FP32 three (GB pair) and four
   (chain rule), in FP64 two (whose wider registers would otherwise lower the
   occupancy) */
template <typename R>
struct SymNI {
  /* FP32: four i atoms, two packed pairs of k_agb_x2 */
  static constexpr int agb = sizeof(R) == 4 ? 4 : 2;
  static constexpr int gbd = sizeof(R) == 4 ? 4 : 2;
  /* resident 128-thread blocks per SM asked of the scalar GB pair pass in
     FP32 (kept for comparison, AGBNP3_PAIR_SCALAR=1) */
  static constexpr int agb_blocks = sizeof(R) == 4 ? 5 : 1;
};
#define AGB_NI (SymNI<R>::agb)

template <typename R>
struct AgbI {
  int ia[AGB_NI];
  R x[AGB_NI], y[AGB_NI], z[AGB_NI], q[AGB_NI], b[AGB_NI], c[AGB_NI];
};
template <typename R>
struct AgbJ {
  R x, y, z, q, b, bi;
  R gx, gy, gz, at;
};
template <typename R>
struct AgbP {
  R e[AGB_NI], gx[AGB_NI], gy[AGB_NI], gz[AGB_NI], at[AGB_NI];
};

template <typename R, bool FULL>
__device__ __forceinline__ void agb_tile(const AgbI<R> &I, AgbJ<R> &J, AgbP<R> &P, int lane, int j0, int a1) {
  #pragma unroll 2
  for (int r = 0; r < 32; r++) {
    if (r > 0) {
      J.x = rot1(J.x); J.y = rot1(J.y); J.z = rot1(J.z);
      J.q = rot1(J.q); J.b = rot1(J.b); J.bi = rot1(J.bi);
    }
    const int jr = j0 + ((lane + r) & 31);
    const bool jok = FULL || jr < a1;
#pragma unroll
    for (int u = 0; u < AGB_NI; u++) {
      R dx = J.x - I.x[u], dy = J.y - I.y[u], dz = J.z - I.z[u];
      R d2 = dx * dx + dy * dy + dz * dz;
      if (!((FULL || (jok && I.ia[u] < jr)) && d2 > R(0))) continue; /* coincident atoms are skipped */
      R bb = I.b[u] * J.b;
      R et = GbExp<R>::ex(I.c[u] * J.bi * d2);
      R f = p_rsqrt(d2 + bb * et);
      R qf = I.q[u] * J.q * f;
      P.e[u] += qf;
      R qf3 = qf * (f * f), eq = et * qf3;
      R mw = qf3 - R(0.25) * eq;
      P.gx[u] = fma(mw, dx, P.gx[u]); P.gy[u] = fma(mw, dy, P.gy[u]); P.gz[u] = fma(mw, dz, P.gz[u]);
      J.gx = fma(-mw, dx, J.gx); J.gy = fma(-mw, dy, J.gy); J.gz = fma(-mw, dz, J.gz);
      R at = eq * (bb + R(0.25) * d2);
      P.at[u] += at;
      J.at += at;
    }
    J.gx = rot1(J.gx); J.gy = rot1(J.gy); J.gz = rot1(J.gz); J.at = rot1(J.at);
  }
}

template <typename R>
__global__ void __launch_bounds__(128, SymNI<R>::agb_blocks) k_agb_sym(View v, const int4 *__restrict__ items, int nitems) {
  const int lane = threadIdx.x & 31;
  const R *X = pa<R>(v, PA_X), *Y = pa<R>(v, PA_Y), *Z = pa<R>(v, PA_Z);
  const R *Q = pa<R>(v, PA_Q), *Bv = pa<R>(v, PA_B), *BI = pa<R>(v, PA_BINV);
  size_t N = v.natoms;
  for (int it = blockIdx.x * 4 + (threadIdx.x >> 5); it < nitems; it += gridDim.x * 4) {
    int4 w = items[it]; /* instance, first atom of the i block, first atom of the j run, j tiles */
    const int a1 = v.inst_begin[w.x + 1];
    const double w2 = 2.0 * v.inst_df[w.x];
    AgbI<R> I;
    AgbP<R> P; /* i-side sums over the run, in R */
#pragma unroll
    for (int u = 0; u < AGB_NI; u++) {
      int i = w.y + 32 * u + lane;
      bool ok = i < a1;
      I.x[u] = ok ? X[i] : R(0);
      I.y[u] = ok ? Y[i] : R(0);
      I.z[u] = ok ? Z[i] : R(0);
      I.q[u] = ok ? Q[i] : R(0);
      I.b[u] = ok ? Bv[i] : R(1);
      I.c[u] = ok ? GbExp<R>::scale() * BI[i] : R(0);
      I.ia[u] = ok ? i : INT_MAX; /* no valid partner: i < j never holds */
      P.e[u] = P.gx[u] = P.gy[u] = P.gz[u] = P.at[u] = R(0);
    }
    const int iend = w.y + 32 * AGB_NI;
    for (int k = 0; k < w.w; k++) {
      const int j0 = w.z + 32 * k;
      const int j = j0 + lane;
      const bool vj = j < a1;
      AgbJ<R> J;
      J.x = vj ? X[j] : R(0);
      J.y = vj ? Y[j] : R(0);
      J.z = vj ? Z[j] : R(0);
      J.q = vj ? Q[j] : R(0);
      J.b = vj ? Bv[j] : R(1);
      J.bi = vj ? BI[j] : R(0);
      J.gx = J.gy = J.gz = J.at = R(0);
      if (iend <= a1 && j0 >= iend && j0 + 32 <= a1) /* warp-uniform */
        agb_tile<R, true>(I, J, P, lane, j0, a1);
      else
        agb_tile<R, false>(I, J, P, lane, j0, a1);
      if (vj) {
        const int ja = v.slot_atom[j];
        atomicAdd(&v.g_gb[3 * ja], w2 * (double)J.gx);
        atomicAdd(&v.g_gb[3 * ja + 1], w2 * (double)J.gy);
        atomicAdd(&v.g_gb[3 * ja + 2], w2 * (double)J.gz);
        atomicAdd(&v.dera[ja], (double)J.at);
      }
    }
#pragma unroll
    for (int u = 0; u < AGB_NI; u++) {
      if (I.ia[u] >= a1) continue;
      const int i = v.slot_atom[I.ia[u]];
      atomicAdd(&v.eatom[N + i], C_TOKCAL * w2 * (double)P.e[u]);
      atomicAdd(&v.g_gb[3 * i], w2 * (double)P.gx[u]);
      atomicAdd(&v.g_gb[3 * i + 1], w2 * (double)P.gy[u]);
      atomicAdd(&v.g_gb[3 * i + 2], w2 * (double)P.gz[u]);
      atomicAdd(&v.dera[i], (double)P.at[u]);
    }
  }
}

/* gbders: both descreening directions of every unordered pair with a heavy
   atom, pair forces, U and V (agbnp3_cpu_simd_kernels.c:681-904).  After
   the heavy-first ordering almost every j tile is interior: all 32 atoms
   valid, after the i block, and all heavy (both directions) or all
   hydrogens (only "j descreened by i"); those tiles run a rotation loop
   without per-pair flags, the table-range test done by selects. */
enum { GBD_GEN = 0, GBD_HH = 1, GBD_HX = 2 };
#define GBD_NI (SymNI<R>::gbd)

template <typename R>
struct GbdI { /* a lane's i atoms */
  int ia[GBD_NI], ti[GBD_NI];
  bool hi[GBD_NI];
  R x[GBD_NI], y[GBD_NI], z[GBD_NI], rh[GBD_NI], sp[GBD_NI], q2[GBD_NI], ab[GBD_NI];
};
template <typename R>
struct GbdJ { /* the j atom a lane holds in a rotation step, and its sums */
  R x, y, z, rh, sp, q2, ab;
  int t;
  R U, V, fx, fy, fz, vx, vy, vz;
};
template <typename R>
struct GbdP { /* i-side sums over one j tile */
  R U[GBD_NI], V[GBD_NI], fx[GBD_NI], fy[GBD_NI], fz[GBD_NI], vx[GBD_NI], vy[GBD_NI], vz[GBD_NI];
};

/* an atom descreened by one of radius R at distance d, rhs = 1/(h R):
   q = Q4/R and dq = d(Q4/R)/dd = (derivative in t) * rhs */
template <typename R, bool SEL, bool REF>
__device__ __forceinline__ bool gbd_q4(const typename Tab<R>::T *tv, int slot, R d, R rhs, R &q, R &dq) {
  R xh = d * rhs;
  if (SEL) { /* no range test: the clamped lookup gives 0 beyond the table */
    R fp;
    q = spline_d<R, REF>(tv, slot, xh, fp);
    dq = fp * rhs;
    return true;
  }
  if (!(xh < R(AGB_NA - 1))) return false;
  R fp;
  q = spline_d<R, REF>(tv, slot, xh, fp);
  dq = fp * rhs;
  return true;
}

template <typename R, int MODE, bool REF>
__device__ __forceinline__ void gbd_tile(const GbdI<R> &I, GbdJ<R> &J, GbdP<R> &P, int lane, int j0, int a1, int hh,
                                         const typename Tab<R>::T *tv, int nt) {
  for (int r = 0; r < 32; r++) {
    if (r > 0) {
      J.x = rot1(J.x); J.y = rot1(J.y); J.z = rot1(J.z);
      J.q2 = rot1(J.q2); J.ab = rot1(J.ab); J.t = rot1(J.t);
      if (MODE != GBD_HX) { /* hydrogens do not descreen: no radius, sp, U, V of j */
        J.rh = rot1(J.rh); J.sp = rot1(J.sp);
      }
    }
    const int jr = j0 + ((lane + r) & 31);
    const bool jok = MODE != GBD_GEN || jr < a1;
    const bool hj = MODE == GBD_HH || (MODE == GBD_GEN && jr < hh);
#pragma unroll
    for (int u = 0; u < GBD_NI; u++) {
      const bool hiu = MODE != GBD_GEN || I.hi[u];
      R dx = J.x - I.x[u], dy = J.y - I.y[u], dz = J.z - I.z[u];
      R d2 = dx * dx + dy * dy + dz * dz;
      R id = p_rsqrt(d2);
      R d = d2 * id;
      if (MODE == GBD_GEN) {
        if (!(jok && I.ia[u] < jr && (hiu || hj) && d2 > R(0))) continue;
      } else {
        /* a step in which no lane's pair is inside the table in either
           direction adds exactly zero: the warp skips it (the vote comes
           before any lane leaves the step) */
        const bool inr = d * I.rh[u] < R(AGB_NA - 1) || (MODE == GBD_HH && d * J.rh < R(AGB_NA - 1));
        if (!__any_sync(0xffffffffu, inr)) continue;
        if (!(d2 > R(0))) continue; /* coincident atoms */
      }
      R ht = R(0), ut = R(0), q, dq;
      if (hiu && gbd_q4<R, MODE != GBD_GEN, REF>(tv, J.t * nt + I.ti[u], d, I.rh[u], q, dq)) {
        /* j descreened by i: table (type j, type i), radius of i */
        P.U[u] += J.q2 * q;
        P.V[u] += J.ab * q;
        ht += J.q2 * dq * I.sp[u];
        ut += J.ab * dq * I.sp[u];
      }
      if (hj && gbd_q4<R, MODE != GBD_GEN, REF>(tv, I.ti[u] * nt + J.t, d, J.rh, q, dq)) {
        /* i descreened by j: table (type i, type j), radius of j */
        J.U += I.q2[u] * q;
        J.V += I.ab[u] * q;
        ht += I.q2[u] * dq * J.sp;
        ut += I.ab[u] * dq * J.sp;
      }
      ht *= id;
      ut *= id;
      P.fx[u] = fma(ht, dx, P.fx[u]); P.fy[u] = fma(ht, dy, P.fy[u]); P.fz[u] = fma(ht, dz, P.fz[u]);
      P.vx[u] = fma(ut, dx, P.vx[u]); P.vy[u] = fma(ut, dy, P.vy[u]); P.vz[u] = fma(ut, dz, P.vz[u]);
      J.fx = fma(-ht, dx, J.fx); J.fy = fma(-ht, dy, J.fy); J.fz = fma(-ht, dz, J.fz);
      J.vx = fma(-ut, dx, J.vx); J.vy = fma(-ut, dy, J.vy); J.vz = fma(-ut, dz, J.vz);
    }
    if (MODE != GBD_HX) {
      J.U = rot1(J.U); J.V = rot1(J.V);
    }
    J.fx = rot1(J.fx); J.fy = rot1(J.fy); J.fz = rot1(J.fz);
    J.vx = rot1(J.vx); J.vy = rot1(J.vy); J.vz = rot1(J.vz);
  }
}

template <typename R, bool REF>
__global__ void __launch_bounds__(128) k_gbders_sym(View v, const int4 *__restrict__ items, int nitems) {
  const int lane = threadIdx.x & 31;
  const R *X = pa<R>(v, PA_X), *Y = pa<R>(v, PA_Y), *Z = pa<R>(v, PA_Z);
  const R *RH = pa<R>(v, PA_RH), *SP = pa<R>(v, PA_SP);
  const R *Q2 = pa<R>(v, PA_Q2AB), *AB = pa<R>(v, PA_ABRW);
  const typename Tab<R>::T *tv = Tab<R>::val(v);
  const int nt = v.ntypes;
  const double f4p = 1.0 / (4.0 * C_PI);
  for (int it = blockIdx.x * 4 + (threadIdx.x >> 5); it < nitems; it += gridDim.x * 4) {
    int4 w = items[it];
    const int a0 = v.inst_begin[w.x], hh = a0 + v.inst_nheavy[w.x], a1 = v.inst_begin[w.x + 1];
    const double kg = f4p * v.inst_df[w.x];
    GbdI<R> I;
    GbdP<R> P; /* i-side sums over the run, in R */
#pragma unroll
    for (int u = 0; u < GBD_NI; u++) {
      int i = w.y + 32 * u + lane;
      bool ok = i < a1;
      I.hi[u] = i < hh;
      I.x[u] = ok ? X[i] : R(0);
      I.y[u] = ok ? Y[i] : R(0);
      I.z[u] = ok ? Z[i] : R(0);
      I.rh[u] = ok ? RH[i] : R(0);
      I.sp[u] = ok ? SP[i] : R(0);
      I.q2[u] = ok ? Q2[i] : R(0);
      I.ab[u] = ok ? AB[i] : R(0);
      I.ti[u] = ok ? v.slot_type[i] : 0;
      I.ia[u] = ok ? i : INT_MAX; /* no valid partner: i < j never holds */
      P.U[u] = P.V[u] = P.fx[u] = P.fy[u] = P.fz[u] = P.vx[u] = P.vy[u] = P.vz[u] = R(0);
    }
    const bool iheavy = w.y + 32 * GBD_NI <= hh; /* every i tile complete and heavy */
    for (int k = 0; k < w.w; k++) {
      const int j0 = w.z + 32 * k;
      const int j = j0 + lane;
      const bool vj = j < a1;
      GbdJ<R> J;
      J.x = vj ? X[j] : R(0);
      J.y = vj ? Y[j] : R(0);
      J.z = vj ? Z[j] : R(0);
      J.rh = vj ? RH[j] : R(0);
      J.sp = vj ? SP[j] : R(0);
      J.q2 = vj ? Q2[j] : R(0);
      J.ab = vj ? AB[j] : R(0);
      J.t = vj ? v.slot_type[j] : 0;
      J.U = J.V = J.fx = J.fy = J.fz = J.vx = J.vy = J.vz = R(0);
      /* warp-uniform tile class */
      const bool interior = iheavy && j0 >= w.y + 32 * GBD_NI;
      if (interior && j0 + 32 <= hh)
        gbd_tile<R, GBD_HH, REF>(I, J, P, lane, j0, a1, hh, tv, nt);
      else if (interior && j0 >= hh && j0 + 32 <= a1)
        gbd_tile<R, GBD_HX, REF>(I, J, P, lane, j0, a1, hh, tv, nt);
      else
        gbd_tile<R, GBD_GEN, REF>(I, J, P, lane, j0, a1, hh, tv, nt);
      if (vj) {
        const int ja = v.slot_atom[j];
        atomicAdd(&v.g_gb[3 * ja], kg * (double)J.fx);
        atomicAdd(&v.g_gb[3 * ja + 1], kg * (double)J.fy);
        atomicAdd(&v.g_gb[3 * ja + 2], kg * (double)J.fz);
        atomicAdd(&v.g_vw[3 * ja], f4p * (double)J.vx);
        atomicAdd(&v.g_vw[3 * ja + 1], f4p * (double)J.vy);
        atomicAdd(&v.g_vw[3 * ja + 2], f4p * (double)J.vz);
        if (j < hh) {
          atomicAdd(&v.deru[ja], (double)J.U);
          atomicAdd(&v.derv[ja], (double)J.V);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < GBD_NI; u++) {
      if (I.ia[u] >= a1) continue;
      const int i = v.slot_atom[I.ia[u]];
      atomicAdd(&v.g_gb[3 * i], kg * (double)P.fx[u]);
      atomicAdd(&v.g_gb[3 * i + 1], kg * (double)P.fy[u]);
      atomicAdd(&v.g_gb[3 * i + 2], kg * (double)P.fz[u]);
      atomicAdd(&v.g_vw[3 * i], f4p * (double)P.vx[u]);
      atomicAdd(&v.g_vw[3 * i + 1], f4p * (double)P.vy[u]);
      atomicAdd(&v.g_vw[3 * i + 2], f4p * (double)P.vz[u]);
      if (I.hi[u]) {
        atomicAdd(&v.deru[i], (double)P.U[u]);
        atomicAdd(&v.derv[i], (double)P.V[u]);
      }
    }
  }
}

#include "agbnp3_pairx2.cuh"

/* U_i, V_i normalised by the atomic volume and the surface-area effective
   gammas (agbnp3_cpu_simd_kernels.c:861-874) */
/* the per-atom values the tree-derivative pass reads for each parent of a
   record, in one record per atom (three or five 16-byte loads instead of
   nine scattered ones): U_i and V_i over the self volume, the cavity, vdW
   and GB weights gammap, dervs, derus, the Gaussian exponent, 1/R and the
   position.  The HB weight derh comes from the water-site stage, which may
   still run beside this kernel, and is read on its own. */
template <typename R>
struct alignas(16) TdAtom {
  double du, dv;
  R wc, wv, wb, ga, gr, x, y, z;
};
static_assert(sizeof(TdAtom<double>) <= 80, "tdat holds 80 bytes per atom");

template <typename R>
__global__ void k_gbders_post(View v) {
  AGB_GRID_STRIDE(g, v.natoms) {
    int I = v.inst_of[g];
    double du = 0.0, dv = 0.0, dvs = 0.0, dus = 0.0;
    if (g < v.inst_begin[I] + v.inst_nheavy[I]) {
      const double f4p = 1.0 / (4.0 * C_PI);
      double vol = v.vols[g];
      du = v.deru[g] / vol;
      dv = v.derv[g] / vol;
      dvs = f4p * v.psvol[g] * dv;
      dus = v.inst_df[I] * f4p * v.psvol[g] * du;
    }
    v.deru[g] = du;
    v.derv[g] = dv;
    v.dervs[g] = dvs;
    v.derus[g] = dus;
    TdAtom<R> t;
    t.du = du;
    t.dv = dv;
    t.wc = (R)v.gammap[g];
    t.wv = (R)dvs;
    t.wb = (R)dus;
    t.ga = atom_alpha<R>(v, g);
    t.gr = atom_rinv<R>(v, g);
    t.x = px<R>(v, g);
    t.y = py<R>(v, g);
    t.z = pz<R>(v, g);
    ((TdAtom<R> *)v.tdat)[g] = t;
  }
}

/* ------------------------------------------------------------------------ */
/* ws: water-site geometry and Jacobians                                    */
/* ------------------------------------------------------------------------ */
template <typename R>
struct V3 {
  R x, y, z;
};
template <typename R>
__device__ __forceinline__ V3<R> vsub(V3<R> a, V3<R> b) {
  return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <typename R>
__device__ __forceinline__ R vnorm(V3<R> a) {
  return m_sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
}
template <typename R>
__device__ __forceinline__ V3<R> vscale(V3<R> a, R s) {
  return {a.x * s, a.y * s, a.z * s};
}
template <typename R>
__device__ __forceinline__ V3<R> vcross(V3<R> a, V3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename R>
__device__ __forceinline__ R vc(V3<R> a, int i) {
  return i == 0 ? a.x : (i == 1 ? a.y : a.z);
}
template <typename R>
__device__ __forceinline__ V3<R> atom_v(const View &v, int g) {
  return {px<R>(v, g), py<R>(v, g), pz<R>(v, g)};
}

/* (I - u u^T) / L : derivative of the unit vector of a vector of length L */
template <typename R>
__device__ __forceinline__ void unit_der(V3<R> u, R invL, R D[3][3]) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) D[i][j] = invL * ((i == j ? R(1) : R(0)) - vc(u, i) * vc(u, j));
}
/* C = A B */
template <typename R>
__device__ __forceinline__ void mmul(const R A[3][3], const R B[3][3], R C[3][3]) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) C[i][j] = A[i][0] * B[0][j] + A[i][1] * B[1][j] + A[i][2] * B[2][j];
}
/* d(a x b)/db (rows: components of a x b) */
template <typename R>
__device__ __forceinline__ void cross_der_b(V3<R> a, R D[3][3]) {
  D[0][0] = 0; D[0][1] = -a.z; D[0][2] = a.y;
  D[1][0] = a.z; D[1][1] = 0; D[1][2] = -a.x;
  D[2][0] = -a.y; D[2][1] = a.x; D[2][2] = 0;
}
/* d(a x b)/da */
template <typename R>
__device__ __forceinline__ void cross_der_a(V3<R> b, R D[3][3]) {
  D[0][0] = 0; D[0][1] = b.z; D[0][2] = -b.y;
  D[1][0] = -b.z; D[1][1] = 0; D[1][2] = b.x;
  D[2][0] = b.y; D[2][1] = -b.x; D[2][2] = 0;
}

template <typename R>
__global__ void k_ws_geom(View v) {
  R *wpos = (R *)v.wpos, *wd = (R *)v.wdpos;
  const R L = R(C_HBLEN);
  AGB_GRID_STRIDE(w, v.nws) {
    const int *P = v.ws_parent + 4 * w;
    int kind = v.ws_kind[w];
    R D[4][3][3];
    for (int p = 0; p < 4; p++)
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) D[p][i][j] = R(0);
    V3<R> pos;
    V3<R> A = atom_v<R>(v, P[0]);
    if (kind == WK_POLARH) { /* parents: hydrogen, heavy atom */
      V3<R> Xd = atom_v<R>(v, P[1]);
      V3<R> b = vsub(A, Xd);
      R len = vnorm(b), s = L / len;
      V3<R> u = vscale(b, R(1) / len);
      pos = {Xd.x + s * b.x, Xd.y + s * b.y, Xd.z + s * b.z};
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          R pr = (i == j ? R(1) : R(0)) - vc(u, i) * vc(u, j);
          D[0][i][j] = s * pr;
          D[1][i][j] = (i == j ? R(1) : R(0)) - s * pr;
        }
    } else if (kind == WK_TRIG1_A || kind == WK_TRIG1_B || kind == WK_TET1) {
      /* anti-parallel to R-Rk, from the acceptor: parents A, R, (R1, R2 | Rk) */
      int pk = kind == WK_TRIG1_A ? 2 : (kind == WK_TRIG1_B ? 3 : 2);
      V3<R> Rr = atom_v<R>(v, P[1]), Rk = atom_v<R>(v, P[pk]);
      V3<R> b = vsub(Rk, Rr);
      R len = vnorm(b);
      V3<R> u = vscale(b, R(1) / len);
      pos = {A.x - L * u.x, A.y - L * u.y, A.z - L * u.z};
      for (int i = 0; i < 3; i++) {
        D[0][i][i] = R(1);
        for (int j = 0; j < 3; j++) {
          R gg = (L / len) * ((i == j ? R(1) : R(0)) - vc(u, i) * vc(u, j));
          D[1][i][j] = gg;
          D[pk][i][j] = -gg;
        }
      }
    } else if (kind == WK_TRIGS_A || kind == WK_TRIGS_B) {
      /* 60 degrees off the R->A axis towards +-(R1-R) x (A-R); parents A, R, R1, R2 */
      const R cth = R(0.5), sth = R(0.866025);
      R sg = kind == WK_TRIGS_A ? R(1) : R(-1);
      V3<R> Rr = atom_v<R>(v, P[1]), R1 = atom_v<R>(v, P[2]);
      V3<R> e0 = vsub(A, Rr), e1 = vsub(R1, Rr);
      R l0 = vnorm(e0);
      V3<R> uin = vscale(e0, R(1) / l0);
      V3<R> n = vcross(e1, e0);
      R ln = vnorm(n);
      V3<R> uout = vscale(n, R(1) / ln);
      pos = {A.x + L * (cth * uin.x + sg * sth * uout.x), A.y + L * (cth * uin.y + sg * sth * uout.y),
             A.z + L * (cth * uin.z + sg * sth * uout.z)};
      R Din[3][3], Dout[3][3], Ce0[3][3], Ce1[3][3], G0[3][3], G1[3][3];
      unit_der(uin, R(1) / l0, Din);
      unit_der(uout, R(1) / ln, Dout);
      cross_der_b(e1, Ce0); /* d(e1 x e0)/de0 */
      cross_der_a(e0, Ce1); /* d(e1 x e0)/de1 */
      mmul(Dout, Ce0, G0);
      mmul(Dout, Ce1, G1);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          R gin = L * cth * Din[i][j], g0 = sg * L * sth * G0[i][j], g1 = sg * L * sth * G1[i][j];
          D[0][i][j] = gin + g0 + (i == j ? R(1) : R(0));
          D[1][i][j] = -gin - g0 - g1;
          D[2][i][j] = g1;
        }
    } else if (kind == WK_OOP_A || kind == WK_OOP_B) {
      /* along +-normal of the R1 R2 R3 plane at 2.7 A; parents A, R1, R2, R3 */
      const R dist = R((float)(C_HBLEN + 0.2));
      R sg = kind == WK_OOP_A ? R(1) : R(-1);
      V3<R> R1 = atom_v<R>(v, P[1]), R2 = atom_v<R>(v, P[2]), R3 = atom_v<R>(v, P[3]);
      V3<R> v1 = vsub(R2, R1), v2 = vsub(R3, R1);
      V3<R> n = vcross(v2, v1);
      R ln = vnorm(n);
      V3<R> nu = vscale(n, R(1) / ln);
      pos = {A.x + sg * dist * nu.x, A.y + sg * dist * nu.y, A.z + sg * dist * nu.z};
      R Pm[3][3], C1[3][3], C2[3][3], G1[3][3], G2[3][3];
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Pm[i][j] = (i == j ? R(1) : R(0)) - vc(nu, i) * vc(nu, j);
      cross_der_b(v2, C1); /* d(v2 x v1)/dv1 */
      cross_der_a(v1, C2); /* d(v2 x v1)/dv2 */
      mmul(Pm, C1, G1);
      mmul(Pm, C2, G2);
      R sc = sg * dist / ln;
      for (int i = 0; i < 3; i++) {
        D[0][i][i] = R(1);
        for (int j = 0; j < 3; j++) {
          D[2][i][j] = sc * G1[i][j];
          D[3][i][j] = sc * G2[i][j];
          D[1][i][j] = -(D[2][i][j] + D[3][i][j]);
        }
      }
    } else if (kind == WK_BIS2 || kind == WK_BIS3) {
      /* opposite the sum of the bond unit vectors; parents A, R1, R2 (, R3) */
      int nb = kind == WK_BIS2 ? 2 : 3;
      V3<R> u[3];
      R inv[3];
      V3<R> s = {R(0), R(0), R(0)};
      for (int q = 0; q < nb; q++) {
        V3<R> b = vsub(atom_v<R>(v, P[q + 1]), A);
        R len = vnorm(b);
        inv[q] = R(1) / len;
        u[q] = vscale(b, inv[q]);
        s.x += u[q].x;
        s.y += u[q].y;
        s.z += u[q].z;
      }
      R ls = vnorm(s);
      V3<R> us = vscale(s, R(1) / ls);
      pos = {A.x - L * us.x, A.y - L * us.y, A.z - L * us.z};
      R Ds[3][3];
      unit_der(us, R(1) / ls, Ds);
      for (int i = 0; i < 3; i++) D[0][i][i] = R(1);
      for (int q = 0; q < nb; q++) {
        R Dq[3][3], G[3][3];
        unit_der(u[q], inv[q], Dq);
        mmul(Ds, Dq, G);
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) {
            D[q + 1][i][j] = -L * G[i][j];
            D[0][i][j] += L * G[i][j];
          }
      }
    } else { /* WK_TET2_A / WK_TET2_B: parents A, R1, R2 */
      const R cth = R(-0.577350269), sth = R(0.816496581);
      R sg = kind == WK_TET2_A ? R(1) : R(-1);
      V3<R> r1 = vsub(atom_v<R>(v, P[1]), A), r2 = vsub(atom_v<R>(v, P[2]), A);
      R l1 = vnorm(r1), l2 = vnorm(r2);
      V3<R> u1 = vscale(r1, R(1) / l1), u2 = vscale(r2, R(1) / l2);
      V3<R> s = {u1.x + u2.x, u1.y + u2.y, u1.z + u2.z};
      R ls = vnorm(s);
      V3<R> uin = vscale(s, R(1) / ls);
      V3<R> n = vcross(r2, r1);
      R ln = vnorm(n);
      V3<R> uout = vscale(n, R(1) / ln);
      pos = {A.x + L * (cth * uin.x + sg * sth * uout.x), A.y + L * (cth * uin.y + sg * sth * uout.y),
             A.z + L * (cth * uin.z + sg * sth * uout.z)};
      R Ds[3][3], D1[3][3], D2[3][3], Gi1[3][3], Gi2[3][3], Do[3][3], C1[3][3], C2[3][3], Go1[3][3], Go2[3][3];
      unit_der(uin, R(1) / ls, Ds);
      unit_der(u1, R(1) / l1, D1);
      unit_der(u2, R(1) / l2, D2);
      mmul(Ds, D1, Gi1);
      mmul(Ds, D2, Gi2);
      unit_der(uout, R(1) / ln, Do);
      cross_der_b(r2, C1); /* d(r2 x r1)/dr1 */
      cross_der_a(r1, C2); /* d(r2 x r1)/dr2 */
      mmul(Do, C1, Go1);
      mmul(Do, C2, Go2);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          R a1 = L * cth * Gi1[i][j] + sg * L * sth * Go1[i][j];
          R a2 = L * cth * Gi2[i][j] + sg * L * sth * Go2[i][j];
          D[1][i][j] = a1;
          D[2][i][j] = a2;
          D[0][i][j] = -(a1 + a2) + (i == j ? R(1) : R(0));
        }
    }
    wpos[3 * w] = pos.x;
    wpos[3 * w + 1] = pos.y;
    wpos[3 * w + 2] = pos.z;
    for (int p = 0; p < 4; p++)
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) wd[(size_t)w * 36 + p * 9 + i * 3 + j] = D[p][i][j];
  }
}

/* ------------------------------------------------------------------------ */
/* ws: free volumes, HB energy and gradient                                 */
/* ------------------------------------------------------------------------ */
/* heavy atoms within 1.6 (r + 1.4) of a water site, one thread per
   (site, neighbour cell) (agbnp3_cpu_simd_kernels.c:2786-2811) */
template <typename R>
__device__ __forceinline__ int ws_cell_scan(const View &v, int w, int c, int *out, int cap) {
  const R *wpos = (const R *)v.wpos;
  int I = v.ws_inst[w];
  R px_ = wpos[3 * w], py_ = wpos[3 * w + 1], pz_ = wpos[3 * w + 2];
  float inv = 1.0f / v.inst_cell[I];
  int cx, cy, cz;
  cell_of((float)px_, (float)py_, (float)pz_, inv, cx, cy, cz);
  int m = 0;
  for_cell(v, I, cx + c % 3 - 1, cy + (c / 3) % 3 - 1, cz + c / 9 - 1, [&](int h, const f4 &b) {
    R dx, dy, dz, rh;
    if constexpr (sizeof(R) == sizeof(float)) { /* the slot record holds the float position and radius */
      dx = b.x - px_;
      dy = b.y - py_;
      dz = b.z - pz_;
      rh = b.w;
    } else {
      dx = px<R>(v, h) - px_;
      dy = py<R>(v, h) - py_;
      dz = pz<R>(v, h) - pz_;
      rh = (R)v.r[h];
    }
    R u = (rh + R(C_HBRAD)) * R(1.6);
    if (dx * dx + dy * dy + dz * dz < u * u) {
      if (out && m < cap) out[m] = h;
      m++;
    }
  });
  return m;
}

/* one thread per (site, neighbour cell), taken direction-major: the lanes
   of a warp are consecutive sites (of nearby parents) looking in the same
   direction, so they mostly walk the same or neighbouring buckets; counts
   and offsets stay in (site, cell) order */
template <typename R>
__global__ void k_ws_count27(View v) {
  AGB_GRID_STRIDE(q, 27LL * v.nws) {
    const int c = (int)(q / v.nws), w = (int)(q % v.nws);
    v.ws_c27[27 * w + c] = ws_cell_scan<R>(v, w, c, NULL, 0);
  }
}

template <typename R>
__global__ void k_ws_emit27(View v) {
  AGB_GRID_STRIDE(q, 27LL * v.nws) {
    const int c = (int)(q / v.nws), w = (int)(q % v.nws);
    int n = v.ws_c27[27 * w + c], o = v.ws_o27[27 * w + c];
    if (n == 0) continue;
    if (o + n > v.cap_wsc) {
      set_err(v, AGB_ERR_WS_CAP);
      continue;
    }
    ws_cell_scan<R>(v, w, c, v.ws_cand + o, n);
  }
}

/* free volumes, HB energy and gradient (agbnp3_cpu_simd_kernels.c:
   2831-2933): the candidates of a site in heavy-atom index order, spe-
   weighted overlaps subtracted until the free volume drops to 60%.  One
   warp per site: the lanes rank-sort the candidates and evaluate their
   overlaps 32 at a time; the subtraction itself then walks those 32 in
   order (values broadcast from their lanes), so the free volume and the
   point where it stops are those of the sequential loop. */
template <typename R>
__global__ void __launch_bounds__(128) k_ws_free(View v) {
  const int lane = threadIdx.x & 31;
  const R *wpos = (const R *)v.wpos, *wd = (const R *)v.wdpos;
  const R vw = R(4.0 / 3.0 * C_PI * C_HBRAD * C_HBRAD * C_HBRAD);
  const R aw = R(C_KFC / (C_HBRAD * C_HBRAD));
  const unsigned below = (1u << lane) - 1u;
  if (v.dc[DC_ERR] & AGB_ERR_WS_CAP) return;
  for (int w = blockIdx.x * 4 + (threadIdx.x >> 5); w < v.nws; w += gridDim.x * 4) {
    const int o = v.ws_o27[27 * w], e = (w + 1 < v.nws) ? v.ws_o27[27 * (w + 1)] : v.dc[DC_WSC];
    const int nc = e - o;
    const int *cand = v.ws_cand + o;
    int *srt = v.ws_srt + o;
    for (int c = lane; c < nc; c += 32) { /* index order; ties keep list order */
      int h = cand[c], rank = 0;
      for (int c2 = 0; c2 < nc; c2++) {
        int h2 = cand[c2];
        rank += (h2 < h) || (h2 == h && c2 < c);
      }
      srt[rank] = h;
    }
    __syncwarp();
    V3<R> p = {wpos[3 * w], wpos[3 * w + 1], wpos[3 * w + 2]};
    const double cut = C_HBSWA0 * (double)vw;
    double fv = (double)vw;
    int prev = v.ws_prev[w];
    double spe_prev = prev >= 0 ? v.spe[prev] : 0.0;
    int np = 0;
    bool done = false;
    for (int c0 = 0; c0 < nc && !done; c0 += 32) {
      const int c = c0 + lane;
      int h = c < nc ? srt[c] : 0;
      double g = 0.0, sh = 0.0;
      if (c < nc) {
        Ov<R> ov = ogauss<R>(aw, R(C_PFC), p.x, p.y, p.z, atom_alpha<R>(v, h), R(C_PFC), px<R>(v, h),
                             py<R>(v, h), pz<R>(v, h));
        if (ov.gvolp > R(0)) {
          g = (double)ov.gvolp;
          sh = v.spe[h];
        }
      }
      unsigned proc = 0;
      const int kend = min(32, nc - c0);
      for (int k = 0; k < kend; k++) {
        double gk = __shfl_sync(0xffffffffu, g, k), sk = __shfl_sync(0xffffffffu, sh, k);
        if (!(fv > cut)) {
          done = true;
          break;
        }
        if (!(gk > 0.0)) continue;
        fv -= (v.compat ? spe_prev : sk) * gk;
        spe_prev = sk;
        proc |= 1u << k;
      }
      __syncwarp();
      if (proc & (1u << lane)) srt[np + __popc(proc & below)] = h; /* processed overlaps, compacted */
      np += __popc(proc);
    }
    __syncwarp();
    double spw = fv / (double)vw, fp, fpp;
    double sw = poly_switch<double>(spw, C_HBSWA, C_HBSWB, fp, fpp);
    double khb = v.ws_khb[w];
    double dhw = khb * fp / (double)vw;
    if (lane == 0) {
      v.ews[w] = khb * sw;
      v.wsp[w] = spw;
    }
    double jw[3] = {0, 0, 0};
    for (int c = lane; c < np; c += 32) {
      int h = srt[c];
      R ah = atom_alpha<R>(v, h);
      Ov<R> ov = ogauss<R>(aw, R(C_PFC), p.x, p.y, p.z, ah, R(C_PFC), px<R>(v, h), py<R>(v, h), pz<R>(v, h));
      double shh = v.spe[h];
      double fi = -2.0 * (double)(ah * ov.gvol * ov.fp), fw = -2.0 * (double)(aw * ov.gvol * ov.fp);
      double uu = -shh * dhw;
      atomicAdd(&v.g_hb[3 * h], uu * fi * (double)(px<R>(v, h) - ov.cx));
      atomicAdd(&v.g_hb[3 * h + 1], uu * fi * (double)(py<R>(v, h) - ov.cy));
      atomicAdd(&v.g_hb[3 * h + 2], uu * fi * (double)(pz<R>(v, h) - ov.cz));
      atomicAdd(&v.derh[h], dhw / v.vols[h] * (double)ov.gvolp);
      jw[0] += uu * fw * (double)(p.x - ov.cx);
      jw[1] += uu * fw * (double)(p.y - ov.cy);
      jw[2] += uu * fw * (double)(p.z - ov.cz);
    }
    for (int off = 16; off > 0; off >>= 1)
      for (int k = 0; k < 3; k++) jw[k] += __shfl_xor_sync(0xffffffffu, jw[k], off);
    /* the site's gradient through its parents: lane 3q+j takes parent q, axis j */
    const int npar = v.ws_nparent[w];
    if (lane < 3 * npar) {
      int q = lane / 3, j = lane % 3;
      int a = v.ws_parent[4 * w + q];
      double t = 0.0;
      for (int k = 0; k < 3; k++) t += jw[k] * (double)wd[(size_t)w * 36 + q * 9 + k * 3 + j];
      atomicAdd(&v.g_hb[3 * a + j], t);
    }
    __syncwarp();
  }
}

/* ------------------------------------------------------------------------ */
/* treeders: derivatives through the self volumes and surface areas         */
/* ------------------------------------------------------------------------ */
/* inclusive sum of a[] over the run of consecutive lanes holding this
   lane's key (a key may come back in a later run, which is summed apart);
   returns whether this lane ends its run */
template <typename T>
__device__ __forceinline__ bool seg_scan12(T (&a)[12], int key) {
  const int lane = threadIdx.x & 31;
  int kp = __shfl_up_sync(0xffffffffu, key, 1);
  int kn = __shfl_down_sync(0xffffffffu, key, 1);
  unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || kp != key);
  int start = 31 - __clz(heads & (0xffffffffu >> (31 - lane))); /* last head at or before this lane */
  const int span = __reduce_max_sync(0xffffffffu, lane - start);      /* longest run in the warp, minus 1 */
  for (int o = 1; o <= span; o <<= 1) {
    bool take = lane - o >= start;
#pragma unroll
    for (int c = 0; c < 12; c++) {
      T t = __shfl_up_sync(0xffffffffu, a[c], o);
      if (take) a[c] += t;
    }
  }
  return lane == 31 || kn != key;
}

/* per record: the contributions to its parents' gradients in the working
   precision (a warp run is at most 32 records), added to the double
   gradients by one atomic per run and component */
template <typename R, int M>
__global__ void __launch_bounds__(256) k_tree_ders(View v) {
  if (v.dc[DC_ERR] & (AGB_ERR_NL_CAP | AGB_ERR_TREE_CAP)) return;
  const int n = min(v.dc[DC_L0 + M], v.cap[M]);
  const int cm = v.cap[M];
  const double f4p = 1.0 / (4.0 * C_PI);
  const double coef = ((M & 1) ? 1.0 : -1.0) / M;
  const double sgn = (M & 1) ? 1.0 : -1.0;
  const int lane = threadIdx.x & 31;
  /* warp-uniform loop: 32 consecutive records per warp step, so that runs of
     records sharing a parent are reduced in the warp before the atomics */
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long base = ((long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < n;
       base += nwarps * 32) {
    const int q = (int)base + lane;
    const bool act = q < n;
    int par[M];
    R gdr[M][3], gdR[M], ga[M], gr[M];
    R wc[M], wv[M], wb[M];
    R su = R(0), sv = R(0), sh = R(0);
    R fp = R(0), h3 = R(0), inva = R(0);
#pragma unroll
    for (int k = 0; k < M; k++) {
      par[k] = act ? v.par[M][(size_t)k * cm + q] : 0;
      gdr[k][0] = gdr[k][1] = gdr[k][2] = R(0);
      gdR[k] = ga[k] = R(0);
      gr[k] = R(1);
      wc[k] = wv[k] = wb[k] = R(0);
    }
    if (act) {
      const Ov<R> o = rec_load<R>(v, M, q);
      R cx = o.cx, cy = o.cy, cz = o.cz, gvol = o.gvol, fpp = o.fpp;
      fp = o.fp;
      inva = f_rcp(o.a);
      double df = v.inst_df[v.inst_of[par[0]]];
      double du = 0.0, dv = 0.0, dh = 0.0;
#pragma unroll
      for (int k = 0; k < M; k++) {
        const int a = par[k];
        const TdAtom<R> t = ((const TdAtom<R> *)v.tdat)[a];
        du += t.du;
        dv += t.dv;
        dh += v.derh[a];
        wc[k] = R(sgn) * t.wc;
        wv[k] = R(sgn) * t.wv;
        wb[k] = R(sgn) * t.wb;
        ga[k] = t.ga;
        gr[k] = t.gr; /* 1/R */
        R u1 = ga[k] * gvol;
        R xk[3] = {t.x - cx, t.y - cy, t.z - cz};
        R d2 = R(0);
#pragma unroll
        for (int c = 0; c < 3; c++) {
          gdr[k][c] = R(-2) * u1 * xk[c];
          d2 += gdr[k][c] * gdr[k][c];
        }
        gdR[k] = (R(3) * inva * u1 + R(0.5) * d2 * f_rcp(u1)) * gr[k];
      }
      su = (R)(du * -df * f4p * coef);
      sv = (R)(dv * -f4p * coef);
      sh = (R)(dh * -coef);
      h3 = fpp + fp * f_rcp(gvol);
    }
    const R h4 = R(2) * fp * inva;
#pragma unroll
    for (int ii = 0; ii < M; ii++) {
      /* gradient on parent ii: gb xyz, vdw xyz, hb xyz, cavity xyz */
      R acc[12];
      R ud = R(-2) * fp * (R(1) - ga[ii] * inva) * gr[ii] + h3 * gdR[ii];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        R ur = gdr[ii][c] * fp;
        R dd = ud * gdr[ii][c];
        acc[c] = su * ur + wb[ii] * dd;
        acc[3 + c] = sv * ur + wv[ii] * dd;
        acc[6 + c] = sh * ur;
        acc[9 + c] = wc[ii] * dd;
      }
#pragma unroll
      for (int jj = 0; jj < M; jj++) {
        if (jj == ii) continue;
        R u1 = h4 * ga[ii] * gr[jj], u2 = h3 * gdR[jj];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          R ur = u1 * gdr[jj][c] + u2 * gdr[ii][c];
          acc[9 + c] += wc[jj] * ur;
          acc[3 + c] += wv[jj] * ur;
          acc[c] += wb[jj] * ur;
        }
      }
      /* parents 0..M-2 are shared by runs of consecutive records (records
         are stored in tree order): sum each run in the warp and let its last
         lane do one atomic per component; the last parent differs from
         record to record */
      int key = act ? par[ii] : -1 - lane;
      bool tail = true;
      if (ii < M - 1) tail = seg_scan12(acc, key);
      if (act && tail) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
          atomicAdd(&v.g_gb[3 * key + c], (double)acc[c]);
          atomicAdd(&v.g_vw[3 * key + c], (double)acc[3 + c]);
          atomicAdd(&v.g_hb[3 * key + c], (double)acc[6 + c]);
          atomicAdd(&v.g_cav[3 * key + c], (double)acc[9 + c]);
        }
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* final: outputs in caller order (agbnp3.c:1761-1786, 537-563)             */
/* ------------------------------------------------------------------------ */
__global__ void k_final(View v) {
  AGB_GRID_STRIDE(g, v.natoms) {
    int e = v.ext_of[g];
    int I = v.inst_of[g];
    bool heavy = g < v.inst_begin[I] + v.inst_nheavy[I];
    v.o_sp[e] = heavy ? v.sp[g] : 1.0;
    v.o_br[e] = v.br[g];
    v.o_sa[e] = heavy ? v.surf_f[g] : 0.0;
    for (int c = 0; c < 3; c++) {
      v.o_gb[3 * e + c] = C_TOKCAL * v.g_gb[3 * g + c];
      v.o_gv[3 * e + c] = v.g_vw[3 * g + c];
      v.o_gc[3 * e + c] = v.g_cav[3 * g + c];
      v.o_gh[3 * e + c] = v.g_hb[3 * g + c];
    }
  }
}

/* per-instance energies from the segment sums: rows of esum are
   eself, epair, evdw, ecorr_vdw, ecav, ecorr_cav, mol_volume (per instance)
   and ehb (per instance) */
__global__ void k_energies(const double *esum, const double *ehb, int ninst, double *out, int *dc) {
  AGB_GRID_STRIDE(I, ninst) {
    double e[7];
    e[0] = esum[I] + esum[ninst + I];
    e[1] = esum[2 * ninst + I];
    e[2] = esum[3 * ninst + I];
    e[3] = esum[4 * ninst + I];
    e[4] = esum[5 * ninst + I];
    e[5] = ehb[I];
    e[6] = esum[6 * ninst + I];
    for (int k = 0; k < 7; k++) {
      out[7 * I + k] = e[k];
      if (!isfinite(e[k])) atomicOr(&dc[DC_ERR], AGB_ERR_NONFINITE);
    }
  }
}

/* ======================================================================== */
/* host side                                                                */
/* ======================================================================== */
static char g_err[512];
#define FAIL(...)                                  \
  do {                                             \
    snprintf(g_err, sizeof(g_err), __VA_ARGS__);   \
    return -1;                                     \
  } while (0)
#define CK(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) FAIL("%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

extern "C" const char *agb_dev_last_error(void) { return g_err; }

/* NCCL, loaded when a sharded instance is first set up (the process may
   already hold the copy its framework loaded, which dlopen then returns) */
static struct {
  int loaded;
  ncclResult_t (*GetUniqueId)(ncclUniqueId *);
  ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int);
  ncclResult_t (*CommDestroy)(ncclComm_t);
  ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t);
  ncclResult_t (*GroupStart)(void);
  ncclResult_t (*GroupEnd)(void);
  const char *(*GetErrorString)(ncclResult_t);
} g_nccl;

static int nccl_load(void) {
  if (g_nccl.loaded) return 0;
  void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
  if (!h) FAIL("NCCL is not available: %s", dlerror());
#define NCCL_SYM(f)                                              \
  do {                                                           \
    *(void **)&g_nccl.f = dlsym(h, "nccl" #f);                   \
    if (!g_nccl.f) FAIL("NCCL has no symbol nccl%s", #f);        \
  } while (0)
  NCCL_SYM(GetUniqueId);
  NCCL_SYM(CommInitRank);
  NCCL_SYM(CommDestroy);
  NCCL_SYM(AllReduce);
  NCCL_SYM(GroupStart);
  NCCL_SYM(GroupEnd);
  NCCL_SYM(GetErrorString);
#undef NCCL_SYM
  g_nccl.loaded = 1;
  return 0;
}


static const char *stage_names[AGB_NSTAGE] = {"prep",  "nblist", "volumes", "scaling", "invb",  "agb",
                                              "gbders", "ws",     "treeders", "final",  "reduce", "spare"};

extern "C" const char *agb_dev_stage_name(int i) { return (i >= 0 && i < AGB_NSTAGE) ? stage_names[i] : ""; }

struct agb_dev {
  int device;
  cudaStream_t st;
  int ninst, natoms, nws, ntypes, precision, compat;
  int *h_inst_begin, *h_ws_begin;
  View v;
  /* owned allocations */
  void *allocs[160];
  int nallocs;
  /* tree capacity (owned separately, regrown on overflow) */
  int cap_nl, cap[AGB_MAX_ORDER + 1], cap_wsc, cap_cand, slab_w;
  float *h_inst_cell; /* each instance's cell edge without a skin */
  int *scan_scratch;
  int scan_cap;
  double *esum, *ehb_inst, *o_energy;
  int *nl_scan_len;
  cudaGraphExec_t gexec;
  int graph_ok;
  int timing;
  cudaEvent_t ev[AGB_NSTAGE + 1];
  cudaStream_t st2;                /* side stream of the water-site stage */
  cudaEvent_t fork_ev, join_ev;    /* orders st2 against st */
  cudaEvent_t tfork_ev, tjoin_ev;  /* the tree-derivative orders split over st and st2 */
  cudaEvent_t xev; /* orders the instance stream against a caller's stream */
  double stage_ms[AGB_NSTAGE];
  long long nlaunch;
  long long last_stats[16];
  int4 *items; /* (instance, first atom, end atom, partner chunk) */
  int nitems, nch;
  int4 *items_agb, *items_gbd; /* (instance, i tile, first j tile, j tiles) */
  int n_agb, n_gbd;
  int tiled_pairs; /* use the one-sided tiled pair kernels instead */
  int scalar_pairs; /* FP32: the scalar symmetric pair kernels instead of the packed f32x2 ones */
  int jb;          /* j tiles per symmetric work item */
  int items_prec;  /* precision the symmetric items were built for (i block size) */
  int *h_inst_nheavy;
  int *h_ext_of;  /* external index of each internal atom */
  /* row sharding of one instance over ranks (one GPU each): this rank's
     share of the pair-stage items, and the communicator that sums the
     pair stages' per-atom partial sums (NULL: emulated, see
     agb_dev_shard_segment) */
  int shard_rank, shard_n;
  ncclComm_t comm;
  int nccl_err;
  int pair_order; /* 1: pair slots along a Hilbert curve, 0: identity */
  size_t gbd_smem;  /* dynamic shared memory of the FP32 chain-rule pass with its tables, 0: tables from global memory */
  size_t desc_smem; /* the same for the FP32 descreening pass */
  int order_ok;   /* the slot order is set for the current mode */
};

static int dev_alloc(agb_dev *s, void **p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) FAIL("cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
  if (s->nallocs >= (int)(sizeof(s->allocs) / sizeof(s->allocs[0]))) FAIL("too many device allocations");
  s->allocs[s->nallocs++] = *p;
  return 0;
}

#define DALLOC(ptr, n, T)                                                        \
  do {                                                                           \
    void *p_;                                                                    \
    if (dev_alloc(s, &p_, (size_t)(n) * sizeof(T)) != 0) return -1;              \
    (ptr) = (T *)p_;                                                             \
  } while (0)

static int upload(void *dst, const void *src, size_t bytes) {
  if (bytes == 0) return 0;
  CK(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
  return 0;
}

static int tree_free(agb_dev *s) {
  for (int m = 2; m <= AGB_MAX_ORDER; m++) {
    if (s->v.par[m]) cudaFree(s->v.par[m]);
    if (s->v.rec[m]) cudaFree(s->v.rec[m]);
    if (s->v.gend[m]) cudaFree(s->v.gend[m]);
    s->v.par[m] = NULL;
    s->v.rec[m] = NULL;
    s->v.gend[m] = NULL;
  }
  for (int m = 2; m <= AGB_MAX_ORDER; m++) {
    if (s->v.lv_cnt[m]) cudaFree(s->v.lv_cnt[m]);
    if (s->v.lv_off[m]) cudaFree(s->v.lv_off[m]);
    if (s->v.lv_mask[m]) cudaFree(s->v.lv_mask[m]);
    if (s->v.lv_own[m]) cudaFree(s->v.lv_own[m]);
    s->v.lv_cnt[m] = s->v.lv_off[m] = s->v.lv_own[m] = NULL;
    s->v.lv_mask[m] = NULL;
  }
  if (s->v.ws_cand) cudaFree(s->v.ws_cand);
  if (s->v.ws_srt) cudaFree(s->v.ws_srt);
  s->v.ws_cand = s->v.ws_srt = NULL;
  if (s->v.nl_list) cudaFree(s->v.nl_list);
  if (s->v.nl_d2) cudaFree(s->v.nl_d2);
  if (s->v.nl_tmp) cudaFree(s->v.nl_tmp);
  if (s->v.nl_own) cudaFree(s->v.nl_own);
  s->v.nl_tmp = s->v.nl_own = NULL;
  if (s->scan_scratch) cudaFree(s->scan_scratch);
  s->v.nl_list = NULL;
  s->v.nl_d2 = NULL;
  s->scan_scratch = NULL;
  int **cand[] = {&s->v.cand_j, &s->v.cand_own, &s->v.cand_flag, &s->v.cand_scan, &s->v.cand_off, &s->v.cand_cnt};
  for (int k = 0; k < 6; k++) {
    if (*cand[k]) cudaFree(*cand[k]);
    *cand[k] = NULL;
  }
  if (s->v.pos_ref) cudaFree(s->v.pos_ref);
  s->v.pos_ref = NULL;
  if (s->v.slab_j) cudaFree(s->v.slab_j);
  if (s->v.slab_d2) cudaFree(s->v.slab_d2);
  s->v.slab_j = NULL;
  s->v.slab_d2 = NULL;
  return 0;
}

static int tree_alloc(agb_dev *s) {
  size_t rsz = sizeof(double); /* records sized for the wider type */
  CK(cudaMalloc((void **)&s->v.ws_cand, sizeof(int) * (size_t)s->cap_wsc));
  CK(cudaMalloc((void **)&s->v.ws_srt, sizeof(int) * (size_t)s->cap_wsc));
  s->v.cap_wsc = s->cap_wsc;
  CK(cudaMalloc((void **)&s->v.nl_list, sizeof(int) * (size_t)s->cap_nl));
  CK(cudaMalloc((void **)&s->v.nl_d2, sizeof(float) * (size_t)s->cap_nl));
  CK(cudaMalloc((void **)&s->v.nl_tmp, sizeof(int) * (size_t)s->cap_nl));
  CK(cudaMalloc((void **)&s->v.nl_own, sizeof(int) * (size_t)s->cap_nl));
  s->v.slab_w = 0;
  if (s->v.skin <= 0.0f) { /* the slabs of the per-evaluation search */
    CK(cudaMalloc((void **)&s->v.slab_j, sizeof(int) * (size_t)s->natoms * 27 * s->slab_w));
    CK(cudaMalloc((void **)&s->v.slab_d2, sizeof(float) * (size_t)s->natoms * 27 * s->slab_w));
    s->v.slab_w = s->slab_w;
  }
  int maxcap = s->natoms;
  for (int m = 2; m <= AGB_MAX_ORDER; m++) {
    CK(cudaMalloc((void **)&s->v.par[m], sizeof(int) * (size_t)m * s->cap[m]));
    CK(cudaMalloc(&s->v.rec[m], rsz * F_NUM * (size_t)s->cap[m]));
    CK(cudaMalloc((void **)&s->v.gend[m], sizeof(int) * (size_t)s->cap[m]));
    if (s->cap[m] > maxcap) maxcap = s->cap[m];
    s->v.cap[m] = s->cap[m];
  }
  /* order 2: one kept flag / offset per near-list entry */
  CK(cudaMalloc((void **)&s->v.lv_cnt[2], sizeof(int) * (size_t)s->cap_nl));
  CK(cudaMalloc((void **)&s->v.lv_off[2], sizeof(int) * (size_t)s->cap_nl));
  for (int m = 3; m <= AGB_MAX_ORDER; m++) {
    /* one count / offset per generating overlap of order m-1 */
    CK(cudaMalloc((void **)&s->v.lv_cnt[m], sizeof(int) * (size_t)s->cap[m - 1]));
    CK(cudaMalloc((void **)&s->v.lv_off[m], sizeof(int) * (size_t)s->cap[m - 1]));
    CK(cudaMalloc((void **)&s->v.lv_mask[m], sizeof(unsigned long long) * (size_t)s->cap[m - 1]));
    CK(cudaMalloc((void **)&s->v.lv_own[m], sizeof(int) * (size_t)s->cap[m]));
  }
  s->scan_cap = maxcap > s->cap_nl ? maxcap : s->cap_nl;
  if (s->v.nbuckets > s->scan_cap) s->scan_cap = s->v.nbuckets;
  if (s->v.sf_nbuckets > s->scan_cap) s->scan_cap = s->v.sf_nbuckets;
  if (27 * s->natoms > s->scan_cap) s->scan_cap = 27 * s->natoms;
  if (27 * s->nws > s->scan_cap) s->scan_cap = 27 * s->nws;
  s->v.cap_cand = 0;
  if (s->v.skin > 0.0f) {
    /* skin candidates; unset build positions force a search at the next
       evaluation */
    const size_t cc = (size_t)s->cap_cand, n = (size_t)s->natoms;
    CK(cudaMalloc((void **)&s->v.cand_j, sizeof(int) * cc));
    CK(cudaMalloc((void **)&s->v.cand_own, sizeof(int) * cc));
    CK(cudaMalloc((void **)&s->v.cand_flag, sizeof(int) * cc));
    CK(cudaMalloc((void **)&s->v.cand_scan, sizeof(int) * cc));
    CK(cudaMalloc((void **)&s->v.cand_off, sizeof(int) * n));
    CK(cudaMalloc((void **)&s->v.cand_cnt, sizeof(int) * n));
    CK(cudaMalloc((void **)&s->v.pos_ref, sizeof(f4) * n));
    CK(cudaMemsetAsync(s->v.pos_ref, 0x7f, sizeof(f4) * n, s->st));
    CK(cudaMemsetAsync(s->v.dc + DC_NCAND, 0, sizeof(int), s->st));
    s->v.cap_cand = s->cap_cand;
    if (s->cap_cand > s->scan_cap) s->scan_cap = s->cap_cand;
  }
  CK(cudaMalloc((void **)&s->scan_scratch, sizeof(int) * ((size_t)s->scan_cap / 1024 + 64)));
  s->v.cap_nl = s->cap_nl;
  return 0;
}

/* pair-stage work lists.  One-sided passes (invb and the tiled fallback):
   tiles of ITILE atoms of one instance, each split into nch partner chunks
   (nch = 0: enough chunks for ~8 blocks per SM).  Symmetric passes: for
   every 32-atom i tile, runs of up to jb j tiles starting at the i tile;
   gbders skips i tiles of hydrogens only (their j tiles are hydrogens too
   and hydrogens never descreen). */
static int build_items(agb_dev *s, int nch, int jb) {
  int NI = s->ninst;
  const int *ib = s->h_inst_begin, *inh = s->h_inst_nheavy;
  int ntiles = 0, maxn = 1;
  for (int I = 0; I < NI; I++) {
    int n = ib[I + 1] - ib[I];
    ntiles += (n + ITILE - 1) / ITILE;
    if (n > maxn) maxn = n;
  }
  if (nch <= 0) {
    /* about 8 items per SM; with the shared-memory tables (one warp per
       half item, 32 warps per SM) about 256, at most 32 chunks */
    const bool sm = s->desc_smem > 0 && s->precision == AGB_PREC_MIXED;
    const int target = sm ? 148 * 256 : 148 * 8;
    nch = (target + ntiles - 1) / ntiles;
    if (sm && nch > 32) nch = 32;
    if (nch > maxn / 512) nch = maxn / 512;
  }
  if (nch < 1) nch = 1;
  if (jb < 1) jb = 1;
  s->nch = nch;
  s->jb = jb;
  /* chunks of about the same length in every instance: the largest
     instance's heavy atoms in nch chunks, a smaller one in fewer (a small
     instance split as finely would spend its items on their set-up) */
  int maxh = 1;
  for (int I = 0; I < NI; I++)
    if (inh[I] > maxh) maxh = inh[I];
  const int clen = (maxh + nch - 1) / nch;
  int *nchi = (int *)malloc(sizeof(int) * (NI > 0 ? NI : 1));
  int nit = 0;
  for (int I = 0; I < NI; I++) {
    int c = (inh[I] + clen - 1) / clen;
    nchi[I] = c < 1 ? 1 : (c > nch ? nch : c);
    nit += ((ib[I + 1] - ib[I] + ITILE - 1) / ITILE) * nchi[I];
  }
  int4 *it = (int4 *)malloc(sizeof(int4) * (nit > 0 ? nit : 1));
  int q = 0;
  for (int I = 0; I < NI; I++)
    for (int a = ib[I]; a < ib[I + 1]; a += ITILE)
      for (int c = 0; c < nchi[I]; c++) {
        int e = a + ITILE < ib[I + 1] ? a + ITILE : ib[I + 1];
        it[q].x = I;
        it[q].y = a;
        it[q].z = e;
        it[q].w = c + 64 * nchi[I]; /* chunk c of nchi[I] (chunk_range) */
        q++;
      }
  free(nchi);
  /* symmetric items: i blocks of SymNI<R> 32-atom tiles for the precision,
     runs of up to jb 32-atom j tiles from the block's first tile to the
     end of the instance */
  const bool f32 = s->precision == AGB_PREC_MIXED;
  const int ni_a = f32 ? SymNI<float>::agb : SymNI<double>::agb, ni_g = f32 ? SymNI<float>::gbd : SymNI<double>::gbd;
  s->items_prec = s->precision;
  int cap_a = 0, cap_g = 0;
  for (int I = 0; I < NI; I++) {
    int T = (ib[I + 1] - ib[I] + 31) / 32;
    for (int tb = 0; tb < T; tb += ni_a) cap_a += (T - tb + jb - 1) / jb;
    for (int tb = 0; tb < T; tb += ni_g) cap_g += (T - tb + jb - 1) / jb;
  }
  int4 *ia = (int4 *)malloc(sizeof(int4) * (cap_a + 1)), *ig = (int4 *)malloc(sizeof(int4) * (cap_g + 1));
  int na = 0, ng = 0;
  for (int I = 0; I < NI; I++) {
    int a0 = ib[I], n = ib[I + 1] - a0, T = (n + 31) / 32;
    int hh = a0 + inh[I];
    for (int pass = 0; pass < 2; pass++) {
      int step = pass == 0 ? ni_a : ni_g;
      for (int tb = 0; tb < T; tb += step)
        for (int tj = tb; tj < T; tj += jb) {
          int4 w;
          w.x = I;
          w.y = a0 + 32 * tb;
          w.z = a0 + 32 * tj;
          w.w = (T - tj) < jb ? (T - tj) : jb;
          if (pass == 0)
            ia[na++] = w;
          else if (w.y < hh) /* blocks of hydrogens only have no gbders pairs */
            ig[ng++] = w;
        }
    }
  }
  if (s->shard_n > 1) {
    /* this rank's share: every shard_n-th item of each list, so that every
       pair is evaluated by exactly one rank and long and short j runs are
       spread over the ranks */
    int4 *L[3] = {it, ia, ig};
    int *cnt[3] = {&nit, &na, &ng};
    for (int k = 0; k < 3; k++) {
      int m = 0;
      for (int q = s->shard_rank; q < *cnt[k]; q += s->shard_n) L[k][m++] = L[k][q];
      *cnt[k] = m;
    }
  }
  if (s->items) cudaFree(s->items);
  if (s->items_agb) cudaFree(s->items_agb);
  if (s->items_gbd) cudaFree(s->items_gbd);
  s->items = s->items_agb = s->items_gbd = NULL;
  CK(cudaMalloc((void **)&s->items, sizeof(int4) * (nit + 1)));
  CK(cudaMalloc((void **)&s->items_agb, sizeof(int4) * (na + 1)));
  CK(cudaMalloc((void **)&s->items_gbd, sizeof(int4) * (ng + 1)));
  if (nit) CK(cudaMemcpy(s->items, it, sizeof(int4) * nit, cudaMemcpyHostToDevice));
  if (na) CK(cudaMemcpy(s->items_agb, ia, sizeof(int4) * na, cudaMemcpyHostToDevice));
  if (ng) CK(cudaMemcpy(s->items_gbd, ig, sizeof(int4) * ng, cudaMemcpyHostToDevice));
  s->nitems = nit;
  s->n_agb = na;
  s->n_gbd = ng;
  free(it);
  free(ia);
  free(ig);
  if (s->graph_ok) {
    cudaGraphExecDestroy(s->gexec);
    s->graph_ok = 0;
  }
  return 0;
}

extern "C" int agb_dev_create(const agb_dev_desc *d, agb_dev **out) {
  *out = NULL;
  if (d->natoms <= 0 || d->ninst <= 0) FAIL("empty system");
  CK(cudaSetDevice(d->device));
  agb_dev *s = (agb_dev *)calloc(1, sizeof(agb_dev));
  if (!s) FAIL("out of host memory");
  s->device = d->device;
  s->ninst = d->ninst;
  s->natoms = d->natoms;
  s->nws = d->nws;
  s->ntypes = d->ntypes;
  s->precision = d->precision;
  s->compat = d->compat;
  CK(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&s->st2, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&s->fork_ev, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&s->join_ev, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&s->tfork_ev, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&s->tjoin_ev, cudaEventDisableTiming));
  View &v = s->v;
  memset(&v, 0, sizeof(v));
  int N = d->natoms, NI = d->ninst, NW = d->nws;
  v.ninst = NI;
  v.natoms = N;
  v.nws = NW;
  v.ntypes = d->ntypes;
  v.compat = d->compat;

  s->h_inst_begin = (int *)malloc(sizeof(int) * (NI + 1));
  s->h_ws_begin = (int *)malloc(sizeof(int) * (NI + 1));
  memcpy(s->h_inst_begin, d->inst_begin, sizeof(int) * (NI + 1));
  memcpy(s->h_ws_begin, d->ws_begin, sizeof(int) * (NI + 1));
  s->h_inst_nheavy = (int *)malloc(sizeof(int) * NI);
  memcpy(s->h_inst_nheavy, d->inst_nheavy, sizeof(int) * NI);

  /* static per-instance data */
  int *inst_of = (int *)malloc(sizeof(int) * N);
  int *bucket_begin = (int *)malloc(sizeof(int) * (NI + 1)), *bucket_mask = (int *)malloc(sizeof(int) * NI);
  int nb = 0, nheavy_tot = 0;
  for (int I = 0; I < NI; I++) {
    for (int g = d->inst_begin[I]; g < d->inst_begin[I + 1]; g++) inst_of[g] = I;
    int want = 2 * d->inst_nheavy[I], sz = 64;
    while (sz < want) sz <<= 1;
    bucket_begin[I] = nb;
    bucket_mask[I] = sz - 1;
    nb += sz;
    nheavy_tot += d->inst_nheavy[I];
  }
  bucket_begin[NI] = nb;
  v.nbuckets = nb;
  int *ws_inst = (int *)malloc(sizeof(int) * (NW > 0 ? NW : 1));
  for (int I = 0; I < NI; I++)
    for (int w = d->ws_begin[I]; w < d->ws_begin[I + 1]; w++) ws_inst[w] = I;
  double *vols = (double *)malloc(sizeof(double) * N);
  for (int g = 0; g < N; g++) vols[g] = 4.0 * C_PI / 3.0 * d->r[g] * d->r[g] * d->r[g];

#define UP(field, src, n, T)                     \
  do {                                           \
    T *p__;                                      \
    DALLOC(p__, (n), T);                         \
    if (upload(p__, (src), sizeof(T) * (size_t)(n))) return -1; \
    v.field = p__;                               \
  } while (0)
  UP(inst_begin, d->inst_begin, NI + 1, int);
  UP(inst_nheavy, d->inst_nheavy, NI, int);
  UP(inst_of, inst_of, N, int);
  UP(inst_df, d->inst_df, NI, double);
  UP(inst_cell, d->inst_cell, NI, float);
  s->h_inst_cell = (float *)malloc(sizeof(float) * NI);
  memcpy(s->h_inst_cell, d->inst_cell, sizeof(float) * NI);
  UP(bucket_begin, bucket_begin, NI + 1, int);
  UP(bucket_mask, bucket_mask, NI, int);
  UP(ext_of, d->ext_of, N, int);
  UP(r, d->r, N, double);
  UP(charge, d->charge, N, double);
  UP(igamma, d->igamma, N, double);
  UP(sgamma, d->sgamma, N, double);
  UP(ialpha, d->ialpha, N, double);
  UP(salpha, d->salpha, N, double);
  UP(vols, vols, N, double);
  UP(rtype, d->rtype, N, int);
  {
    /* per interval k, from the node values y and second derivatives y2 of
       the spline in a (step h), with t = a/h - k:
         f(t) = c0 + c1 t + c2 t^2 + c3 t^3,
         c0 = y_k,  c1 = y_k+1 - y_k - h^2 (2 y2_k + y2_k+1) / 6,
         c2 = h^2 y2_k / 2,  c3 = h^2 (y2_k+1 - y2_k) / 6.
       The coefficients are divided by the radius R of the descreening
       type (the second index of a table), which every atom of that type
       shares.  The last node's record is never read: a lookup stops below
       node AGB_NA-1. */
    const int nt = d->ntypes;
    double *rt = (double *)malloc(sizeof(double) * (nt > 0 ? nt : 1));
    for (int t = 0; t < nt; t++) rt[t] = 0.0;
    for (int g = 0; g < N; g++) {
      int t = d->rtype[g];
      if (rt[t] == 0.0) rt[t] = d->r[g];
      if (rt[t] != d->r[g]) {
        free(rt);
        FAIL("atoms %d of radius type %d have radius %.17g, the type %.17g", g, t, d->r[g], rt[t]);
      }
    }
    size_t nrec = (size_t)nt * nt * AGB_NA;
    double *tv = (double *)calloc(nrec * 4, sizeof(double));
    float *fv = (float *)calloc(nrec * 4, sizeof(float));
    const double h = C_AMAX / (AGB_NA - 1), hh6 = h * h / 6.0;
    for (size_t q = 0; q < nrec; q++) {
      if ((int)(q % AGB_NA) == AGB_NA - 1) continue;
      const double rs = rt[(q / AGB_NA) % nt];
      const double *a = d->tab + q * 2; /* y_k, y2_k, y_k+1, y2_k+1 */
      double c[4] = {a[0], a[2] - a[0] - hh6 * (2.0 * a[1] + a[3]), 0.5 * h * h * a[1], hh6 * (a[3] - a[1])};
      for (int k = 0; k < 4; k++) {
        tv[4 * q + k] = rs > 0.0 ? c[k] / rs : 0.0;
        fv[4 * q + k] = (float)tv[4 * q + k];
      }
    }
    free(rt);
    UP(tabv_d, (const double4 *)tv, nrec, double4);
    UP(tabv_f, (const float4 *)fv, nrec, float4);
    /* the tables of the descreener types that heavy atoms have (hydrogens
       descreen nothing), compacted for the chain-rule pass's shared memory */
    int *hv = (int *)calloc(nt > 0 ? nt : 1, sizeof(int));
    int nhv = 0;
    for (int I = 0; I < NI; I++)
      for (int g = d->inst_begin[I]; g < d->inst_begin[I] + d->inst_nheavy[I]; g++) hv[d->rtype[g]] = 1;
    for (int t = 0; t < nt; t++) hv[t] = hv[t] ? nhv++ : -1;
    size_t nrh = (size_t)nt * (nhv > 0 ? nhv : 1) * AGB_NA;
    float *fh = (float *)calloc(nrh * 4, sizeof(float));
    for (int a = 0; a < nt; a++)
      for (int b = 0; b < nt; b++)
        if (hv[b] >= 0)
          memcpy(fh + 4 * ((size_t)(a * nhv + hv[b]) * AGB_NA), fv + 4 * ((size_t)(a * nt + b) * AGB_NA),
                 sizeof(float) * 4 * AGB_NA);
    for (int t = 0; t < nt; t++) hv[t] = hv[t] < 0 ? 0 : hv[t];
    v.nhv = nhv;
    {
      /* the chain-rule pass holds these tables in shared memory when they
         fit beside its 16 warps' j tiles */
      int smax = 0;
      CK(cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, d->device));
      const size_t need = sizeof(float4) * ((size_t)16 * 4 * 32 + (size_t)nt * nhv * AGB_NA);
      const char *e = getenv("AGBNP3_GBD_SMEM");
      s->gbd_smem = 0;
      if (nhv > 0 && need <= (size_t)smax && (!e || atoi(e) != 0)) {
        CK(cudaFuncSetAttribute(k_gbders_x2<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need));
        CK(cudaFuncSetAttribute(k_gbders_x2<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need));
        s->gbd_smem = need;
      }
      const size_t dneed = sizeof(float4) * ((size_t)DS_WARPS * DS_GROUP * 3 / 2 + (size_t)nt * nhv * AGB_NA);
      const char *e2 = getenv("AGBNP3_DESC_SMEM");
      s->desc_smem = 0;
      if (nhv > 0 && dneed <= (size_t)smax && (!e2 || atoi(e2) != 0)) {
        CK(cudaFuncSetAttribute(k_descreen_s, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dneed));
        s->desc_smem = dneed;
      }
    }
    UP(tabh_f, (const float4 *)fh, nrh, float4);
    UP(hvslot, hv, nt > 0 ? nt : 1, int);
    free(fh);
    free(hv);
    free(tv);
    free(fv);
  }
  {
    /* the surrogate's grid over all atoms: >= 2 buckets per atom */
    int *sbb = (int *)malloc(sizeof(int) * (NI + 1)), *sbm = (int *)malloc(sizeof(int) * NI), snb = 0;
    for (int I = 0; I < NI; I++) {
      int want = 2 * (d->inst_begin[I + 1] - d->inst_begin[I]), sz = 64;
      while (sz < want) sz <<= 1;
      sbb[I] = snb;
      sbm[I] = sz - 1;
      snb += sz;
    }
    sbb[NI] = snb;
    v.sf_nbuckets = snb;
    UP(sf_bbegin, sbb, NI + 1, int);
    UP(sf_bmask, sbm, NI, int);
    DALLOC(v.sf_bcount, snb, int);
    DALLOC(v.sf_bstart, snb, int);
    DALLOC(v.sf_bcursor, snb, int);
    DALLOC(v.sf_abucket, N > 0 ? N : 1, int);
    DALLOC(v.sf_spos, N > 0 ? N : 1, f4);
    DALLOC(v.sf_sid, N > 0 ? N : 1, int2);
    DALLOC(v.sf_dc, 2, int);
    if (upload(v.sf_dc, &snb, sizeof(int))) return -1;
    free(sbb);
    free(sbm);
    signed char *cls = (signed char *)malloc(N > 0 ? N : 1);
    memset(cls, 0xff, N > 0 ? N : 1);
    UP(sclass, cls, N, signed char);
    free(cls);
  }
  UP(ws_begin, d->ws_begin, NI + 1, int);
  if (NW > 0) {
    UP(ws_inst, ws_inst, NW, int);
    UP(ws_kind, d->ws_kind, NW, int);
    UP(ws_parent, d->ws_parent, 4 * NW, int);
    UP(ws_nparent, d->ws_nparent, NW, int);
    UP(ws_prev, d->ws_prev, NW, int);
    UP(ws_khb, d->ws_khb, NW, double);
  }
  free(inst_of);
  free(bucket_begin);
  free(bucket_mask);
  free(ws_inst);
  free(vols);

  /* per-evaluation buffers */
  DALLOC(v.x_ext, N, double);
  DALLOC(v.y_ext, N, double);
  DALLOC(v.z_ext, N, double);
  DALLOC(v.pos, N, f4);
  DALLOC(v.pxd, N, double);
  DALLOC(v.pyd, N, double);
  DALLOC(v.pzd, N, double);
  DALLOC(v.atom_cell, 3 * N, int);
  DALLOC(v.atom_bucket, N, int);
  DALLOC(v.bucket_count, nb, int);
  DALLOC(v.bucket_start, nb, int);
  DALLOC(v.bucket_cursor, nb, int);
  DALLOC(v.cell_pos, N, f4);
  DALLOC(v.cell_id, N, int2);
  DALLOC(v.nl_count, N, int);
  DALLOC(v.nl_off, N, int);
  DALLOC(v.nl_c27, 27 * N, int);
  DALLOC(v.nl_o27, 27 * N, int);
  DALLOC(v.ws_c27, 27 * (NW > 0 ? NW : 1), int);
  DALLOC(v.ws_o27, 27 * (NW > 0 ? NW : 1), int);
  DALLOC(v.dc, DC_SIZE, int);
  double **dbl[] = {&v.volumep, &v.surf, &v.surf_f, &v.sp, &v.spe, &v.psvol, &v.gammap, &v.bfil, &v.bder,
                    &v.br, &v.brw, &v.dera, &v.q2ab, &v.abrw, &v.deru, &v.derv, &v.derh, &v.derus, &v.dervs,
                    &v.o_sp, &v.o_br, &v.o_sa};
  for (size_t k = 0; k < sizeof(dbl) / sizeof(dbl[0]); k++) DALLOC(*dbl[k], N, double);
  {
    void *p;
    if (dev_alloc(s, &p, (size_t)N * 80)) return -1; /* sizeof(TdAtom<double>) */
    v.tdat = p;
  }
  DALLOC(v.g_gb, 3 * N, double);
  DALLOC(v.g_vw, 3 * N, double);
  DALLOC(v.g_cav, 3 * N, double);
  DALLOC(v.g_hb, 3 * N, double);
  DALLOC(v.o_gb, 3 * N, double);
  DALLOC(v.o_gv, 3 * N, double);
  DALLOC(v.o_gc, 3 * N, double);
  DALLOC(v.o_gh, 3 * N, double);
  DALLOC(v.eatom, 7 * N, double);
  DALLOC(v.acc_beta, N, double);
  DALLOC(v.tbox, 2 * ((N + 31) / 32), float4);
  for (int k = 0; k < PA_NUM; k++) {
    void *p;
    if (dev_alloc(s, &p, sizeof(double) * (size_t)N)) return -1;
    v.pa[k] = p;
  }
  {
    /* pair slots: the identity until the first evaluation orders them */
    int *id = (int *)malloc(sizeof(int) * N);
    for (int g = 0; g < N; g++) id[g] = g;
    UP(slot_atom, id, N, int);
    UP(atom_slot, id, N, int);
    free(id);
    DALLOC(v.slot_type, N, int);
    DALLOC(v.slot_hvcol, N, int);
    s->h_ext_of = (int *)malloc(sizeof(int) * N);
    memcpy(s->h_ext_of, d->ext_of, sizeof(int) * N);
    const char *po = getenv("AGBNP3_PAIR_ORDER");
    s->pair_order = po ? atoi(po) != 0 : 1;
    s->order_ok = !s->pair_order;
  }
  {
    const char *tp = getenv("AGBNP3_PAIR_TILED");
    s->tiled_pairs = tp && atoi(tp) != 0;
    const char *sp = getenv("AGBNP3_PAIR_SCALAR");
    s->scalar_pairs = sp && atoi(sp) != 0;
    int nch = 0, jb = 8;
    const char *e1 = getenv("AGBNP3_DESC_CHUNKS"), *e2 = getenv("AGBNP3_SYM_RUN");
    if (e1) nch = atoi(e1);
    if (e2) jb = atoi(e2);
    if (build_items(s, nch, jb)) return -1;
  }

  DALLOC(v.ews, NW > 0 ? NW : 1, double);
  DALLOC(v.wsp, NW > 0 ? NW : 1, double);
  {
    void *p;
    if (dev_alloc(s, &p, sizeof(double) * 3 * (size_t)(NW > 0 ? NW : 1))) return -1;
    v.wpos = p;
    if (dev_alloc(s, &p, sizeof(double) * 36 * (size_t)(NW > 0 ? NW : 1))) return -1;
    v.wdpos = p;
  }
  DALLOC(s->esum, 7 * NI, double);
  DALLOC(s->ehb_inst, NI, double);
  DALLOC(s->o_energy, 7 * NI, double);

  int dc0[DC_SIZE];
  memset(dc0, 0, sizeof(dc0));
  dc0[DC_N] = N;
  dc0[DC_N27] = 27 * N;
  dc0[DC_NB] = nb;
  dc0[DC_NWS] = NW;
  dc0[DC_W27] = 27 * NW;
  if (upload(v.dc, dc0, sizeof(dc0))) return -1;

  /* capacities: kept overlaps per heavy atom at 0.05 atoms/A^3 are ~13,
     28, 19, 5 for orders 2..5 and ~24 near neighbours; start at a few
     times that and grow on overflow */
  s->cap_nl = 48 * nheavy_tot + 4096;
  s->cap[2] = 32 * nheavy_tot + 4096;
  s->cap[3] = 64 * nheavy_tot + 4096;
  s->cap[4] = 64 * nheavy_tot + 4096;
  s->cap[5] = 32 * nheavy_tot + 4096;
  s->cap_wsc = 64 * NW + 1024;
  s->slab_w = 8; /* ~29 near partners j > i per heavy atom on average, over 27 cells */
  /* the near-list search: one thread per (atom, neighbour cell) is faster
     up to a few hundred thousand atoms (measured: 0.104 against 0.120 ms at
     25,000 atoms, 0.400 against 0.425 ms for 207,000 atoms in 128
     instances), one warp per 32 grid slots and direction beyond (1.78
     against 1.49 ms for 827,000 atoms in 512 instances) */
  v.nl_cells = N >= 400000;
  {
    const char *e = getenv("AGBNP3_NL_CELLS"); /* 0 / 1: either search, for tests */
    if (e) v.nl_cells = atoi(e) != 0;
  }
  /* AGBNP3_CAPACITY_SCALE (< 1) starts from smaller buffers, which
     exercises the overflow detection and regrowth of agb_dev_evaluate */
  const char *cs = getenv("AGBNP3_CAPACITY_SCALE");
  if (cs && atof(cs) > 0.0) {
    double f = atof(cs);
    s->cap_nl = (int)(s->cap_nl * f) + 1;
    for (int m = 2; m <= AGB_MAX_ORDER; m++) s->cap[m] = (int)(s->cap[m] * f) + 1;
    s->cap_wsc = (int)(s->cap_wsc * f) + 1;
    s->slab_w = (int)(s->slab_w * f) + 1;
  }
  if (tree_alloc(s)) return -1;
  for (int k = 0; k <= AGB_NSTAGE; k++) CK(cudaEventCreate(&s->ev[k]));
  CK(cudaEventCreateWithFlags(&s->xev, cudaEventDisableTiming));
  *out = s;
  return 0;
}

extern "C" void agb_dev_destroy(agb_dev *s) {
  if (!s) return;
  cudaSetDevice(s->device);
  cudaStreamSynchronize(s->st);
  if (s->graph_ok) cudaGraphExecDestroy(s->gexec);
  if (s->comm) g_nccl.CommDestroy(s->comm);
  tree_free(s);
  for (int k = 0; k < s->nallocs; k++) cudaFree(s->allocs[k]);
  for (int k = 0; k <= AGB_NSTAGE; k++)
    if (s->ev[k]) cudaEventDestroy(s->ev[k]);
  if (s->fork_ev) cudaEventDestroy(s->fork_ev);
  if (s->join_ev) cudaEventDestroy(s->join_ev);
  if (s->tfork_ev) cudaEventDestroy(s->tfork_ev);
  if (s->tjoin_ev) cudaEventDestroy(s->tjoin_ev);
  if (s->st2) cudaStreamDestroy(s->st2);
  if (s->xev) cudaEventDestroy(s->xev);
  cudaStreamDestroy(s->st);
  if (s->items) cudaFree(s->items);
  if (s->items_agb) cudaFree(s->items_agb);
  if (s->items_gbd) cudaFree(s->items_gbd);
  free(s->h_inst_begin);
  free(s->h_ws_begin);
  free(s->h_inst_nheavy);
  free(s->h_ext_of);
  free(s->h_inst_cell);
  free(s);
}

/* Hilbert index of a point of 3 coordinates of `bits` bits each: J. Skilling,
   "Programming the Hilbert curve", AIP Conf. Proc. 707 (2004) -- the axes
   are turned into the transposed index in place, whose bits are then
   interleaved, most significant first. */
static unsigned long long hilbert3(unsigned int X[3], int bits) {
  const unsigned int M = 1u << (bits - 1);
  for (unsigned int Q = M; Q > 1; Q >>= 1) {
    const unsigned int P = Q - 1;
    for (int i = 0; i < 3; i++) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        unsigned int t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  for (int i = 1; i < 3; i++) X[i] ^= X[i - 1];
  unsigned int t = 0;
  for (unsigned int Q = M; Q > 1; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1;
  for (int i = 0; i < 3; i++) X[i] ^= t;
  unsigned long long h = 0;
  for (int b = bits - 1; b >= 0; b--)
    for (int i = 0; i < 3; i++) h = (h << 1) | ((X[i] >> b) & 1u);
  return h;
}

struct slot_key {
  unsigned long long key;
  int g;
};
static int slot_key_cmp(const void *a, const void *b) {
  const slot_key *p = (const slot_key *)a, *q = (const slot_key *)b;
  if (p->key != q->key) return p->key < q->key ? -1 : 1;
  return (p->g > q->g) - (p->g < q->g);
}

/* Pair slots from the coordinates staged for the next evaluation: within
   each instance the heavy atoms keep slots [begin, begin + nheavy) and the
   hydrogens the rest, each group sorted by the Hilbert index of its atoms
   on a 2^10 grid over the instance's bounding cube (ties by atom).  The
   order only changes which atoms share a 32-atom tile of the pair passes
   (and so the summation order); any order gives the same pairs. */
static int order_pair_slots(agb_dev *s) {
  const int N = s->natoms;
  CK(cudaStreamSynchronize(s->st));
  double *xyz = (double *)malloc(sizeof(double) * 3 * (size_t)N);
  int *sa = (int *)malloc(sizeof(int) * N), *as = (int *)malloc(sizeof(int) * N);
  slot_key *keys = (slot_key *)malloc(sizeof(slot_key) * N);
  if (!xyz || !sa || !as || !keys) {
    free(xyz); free(sa); free(as); free(keys);
    FAIL("out of host memory");
  }
  int rc = 0;
  if (cudaMemcpy(xyz, s->v.x_ext, sizeof(double) * N, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(xyz + N, s->v.y_ext, sizeof(double) * N, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(xyz + 2 * (size_t)N, s->v.z_ext, sizeof(double) * N, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = -1;
  const int bits = 10, top = (1 << bits) - 1;
  for (int I = 0; I < s->ninst && rc == 0; I++) {
    const int a0 = s->h_inst_begin[I], hh = a0 + s->h_inst_nheavy[I], a1 = s->h_inst_begin[I + 1];
    double lo[3] = {0.0, 0.0, 0.0}, hi[3] = {0.0, 0.0, 0.0};
    bool first = true;
    for (int g = a0; g < a1; g++) {
      double p[3];
      for (int c = 0; c < 3; c++) p[c] = xyz[(size_t)c * N + s->h_ext_of[g]];
      if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) continue;
      for (int c = 0; c < 3; c++) {
        if (first || p[c] < lo[c]) lo[c] = p[c];
        if (first || p[c] > hi[c]) hi[c] = p[c];
      }
      first = false;
    }
    double ext = fmax(hi[0] - lo[0], fmax(hi[1] - lo[1], hi[2] - lo[2]));
    const double sc = ext > 0.0 ? top / ext : 0.0;
    const int grp[3] = {a0, hh, a1};
    for (int k = 0; k < 2; k++) {
      int n = 0;
      for (int g = grp[k]; g < grp[k + 1]; g++) {
        unsigned int X[3];
        for (int c = 0; c < 3; c++) {
          double q = (xyz[(size_t)c * N + s->h_ext_of[g]] - lo[c]) * sc;
          X[c] = q >= 0.0 && q <= (double)top ? (unsigned int)q : (q > (double)top ? (unsigned int)top : 0u);
        }
        keys[n].key = hilbert3(X, bits);
        keys[n].g = g;
        n++;
      }
      qsort(keys, n, sizeof(slot_key), slot_key_cmp);
      for (int q = 0; q < n; q++) {
        sa[grp[k] + q] = keys[q].g;
        as[keys[q].g] = grp[k] + q;
      }
    }
  }
  if (rc == 0 && (upload((void *)s->v.slot_atom, sa, sizeof(int) * N) ||
                  upload((void *)s->v.atom_slot, as, sizeof(int) * N)))
    rc = -1;
  free(xyz); free(sa); free(as); free(keys);
  if (rc) FAIL("pair slot order: %s", cudaGetErrorString(cudaGetLastError()));
  s->order_ok = 1;
  return 0;
}

extern "C" int agb_dev_set_skin(agb_dev *s, double skin) {
  CK(cudaSetDevice(s->device));
  if (!(skin >= 0.0 && skin <= 10.0)) FAIL("near-list skin %g outside [0, 10] A", skin);
  CK(cudaStreamSynchronize(s->st));
  if (s->graph_ok) {
    cudaGraphExecDestroy(s->gexec);
    s->graph_ok = 0;
  }
  tree_free(s);
  s->v.skin = (float)skin;
  if (skin > 0.0 && s->cap_cand == 0) {
    /* the shell of width skin around the ~5.5 A cutoff adds candidates */
    double f = 1.0 + skin / 5.0;
    s->cap_cand = (int)(f * f * f * s->cap_nl) + 4096;
  }
  /* the cell grid must cover the candidate cutoff */
  float *cell = (float *)malloc(sizeof(float) * s->ninst);
  if (!cell) FAIL("out of host memory");
  for (int I = 0; I < s->ninst; I++) cell[I] = s->h_inst_cell[I] + (float)skin;
  int rc = upload((void *)s->v.inst_cell, cell, sizeof(float) * s->ninst);
  free(cell);
  if (rc) return -1;
  return tree_alloc(s);
}

/* mode 1: order the pair slots along a Hilbert curve from the coordinates
   of the next evaluation (again on each call); mode 0: the identity */
extern "C" int agb_dev_set_pair_order(agb_dev *s, int mode) {
  CK(cudaSetDevice(s->device));
  if (mode != 0 && mode != 1) FAIL("unknown pair order %d", mode);
  s->pair_order = mode;
  if (mode == 1) {
    s->order_ok = 0;
    return 0;
  }
  CK(cudaStreamSynchronize(s->st));
  int *id = (int *)malloc(sizeof(int) * s->natoms);
  if (!id) FAIL("out of host memory");
  for (int g = 0; g < s->natoms; g++) id[g] = g;
  int rc = upload((void *)s->v.slot_atom, id, sizeof(int) * s->natoms) ||
           upload((void *)s->v.atom_slot, id, sizeof(int) * s->natoms);
  free(id);
  if (rc) return -1;
  s->order_ok = 1;
  return 0;
}

extern "C" int agb_dev_set_mode(agb_dev *s, int precision, int compat) {
  if (precision != AGB_PREC_FP64 && precision != AGB_PREC_MIXED) FAIL("unknown precision mode %d", precision);
  if (s->graph_ok && (precision != s->precision || (compat != 0) != (s->compat != 0))) {
    cudaGraphExecDestroy(s->gexec);
    s->graph_ok = 0;
  }
  s->precision = precision;
  s->compat = compat != 0;
  s->v.compat = s->compat;
  if (s->items_agb && s->items_prec != precision && build_items(s, s->nch, s->jb)) return -1;
  return 0;
}

extern "C" int agb_dev_upload_coords(agb_dev *s, const double *x, const double *y, const double *z) {
  CK(cudaSetDevice(s->device));
  size_t b = sizeof(double) * s->natoms;
  CK(cudaMemcpyAsync((void *)s->v.x_ext, x, b, cudaMemcpyHostToDevice, s->st));
  CK(cudaMemcpyAsync((void *)s->v.y_ext, y, b, cudaMemcpyHostToDevice, s->st));
  CK(cudaMemcpyAsync((void *)s->v.z_ext, z, b, cudaMemcpyHostToDevice, s->st));
  return 0;
}

static inline int nblocks(long long n) {
  long long b = (n + BLK - 1) / BLK;
  if (b < 1) b = 1;
  if (b > 148 * 64) b = 148 * 64;
  return (int)b;
}

/* blocks of 4 warps, one work item per warp */
static inline int sym_grid(int n) {
  int b = (n + 3) / 4;
  if (b > 148 * 16) b = 148 * 16;
  return b < 1 ? 1 : b;
}

/* the water-site stage on `stream` */
template <typename R>
static void launch_ws(agb_dev *s, const View &v, cudaStream_t stream) {
  AGB_LAUNCH(k_ws_geom<R>, nblocks(s->nws), BLK, stream, v);
  AGB_LAUNCH(k_ws_count27<R>, nblocks(27LL * s->nws), BLK, stream, v);
  agb_scan_excl(v.ws_c27, v.ws_o27, v.dc + DC_W27, v.dc + DC_WSC, 27 * s->nws, s->scan_scratch, stream);
  AGB_LAUNCH(k_ws_emit27<R>, nblocks(27LL * s->nws), BLK, stream, v);
  AGB_LAUNCH(k_ws_free<R>, sym_grid(s->nws), 128, stream, v);
}

/* the FP32 chain-rule pass: a block on every SM, of as many warps (up to
   16) as the items fill, with the heavy-descreener tables in shared memory
   when they fit, else read from global memory */
static void launch_gbders_x2(agb_dev *s, cudaStream_t st) {
  const View &v = s->v;
  const int grid = s->n_gbd > 148 ? 148 : (s->n_gbd < 1 ? 1 : s->n_gbd);
  int nw = (s->n_gbd + 147) / 148;
  nw = nw > 16 ? 16 : (nw < 1 ? 1 : nw);
  const size_t shb = s->gbd_smem > 0 ? s->gbd_smem : sizeof(float4) * 16 * 4 * 32;
  if (s->gbd_smem > 0 && s->compat)
    k_gbders_x2<true, true><<<grid, nw * 32, shb, st>>>(v, s->items_gbd, s->n_gbd);
  else if (s->gbd_smem > 0)
    k_gbders_x2<false, true><<<grid, nw * 32, shb, st>>>(v, s->items_gbd, s->n_gbd);
  else if (s->compat)
    k_gbders_x2<true, false><<<grid, nw * 32, shb, st>>>(v, s->items_gbd, s->n_gbd);
  else
    k_gbders_x2<false, false><<<grid, nw * 32, shb, st>>>(v, s->items_gbd, s->n_gbd);
}

static void stage_mark(agb_dev *s, int k) {
  if (s->timing) cudaEventRecord(s->ev[k], s->st);
}

/* the whole evaluation as a fixed launch sequence */
/* the per-atom partial sums of pair stage k (0 descreening, 1 GB pair,
   2 chain rule) that a row-sharded evaluation adds over the ranks before
   the next stage reads them; returns how many arrays */
static int shard_bufs(agb_dev *s, int k, double **ptr, size_t *cnt) {
  const size_t N = (size_t)s->natoms;
  View &v = s->v;
  if (k == 0) {
    ptr[0] = v.acc_beta, cnt[0] = N;
    return 1;
  }
  if (k == 1) {
    ptr[0] = v.dera, cnt[0] = N;
    return 1;
  }
  /* the pair energy row of eatom, the constant-volume gradients and U, V;
     nothing else has written these since they were zeroed */
  ptr[0] = v.deru, cnt[0] = N;
  ptr[1] = v.derv, cnt[1] = N;
  ptr[2] = v.g_gb, cnt[2] = 3 * N;
  ptr[3] = v.g_vw, cnt[3] = 3 * N;
  ptr[4] = v.eatom + N, cnt[4] = N;
  return 5;
}

static void shard_allreduce(agb_dev *s, int k, cudaStream_t st);

/* the whole evaluation as a fixed launch sequence; seg >= 0 launches only
   segment seg (0: up to the descreening sums, 1: Born radii and the GB pair
   pass, 2: q2ab/abrw and the chain-rule pass, 3: the rest), between which a
   row-sharded evaluation sums the pair stages' partial sums over the ranks */
template <typename R>
static void launch_all(agb_dev *s, int seg = -1) {
  View v = s->v;
  cudaStream_t st = s->st;
  int N = s->natoms;
  long long nl = 0;
  /* the water-site stage on a side stream (captured whole evaluations) */
  const bool side = !s->timing && s->nws > 0 && seg < 0;
  if (seg < 0 || seg == 0) {
  stage_mark(s, 0);
  cudaMemsetAsync(v.bucket_count, 0, sizeof(int) * v.nbuckets, st);
  cudaMemsetAsync(v.bucket_cursor, 0, sizeof(int) * v.nbuckets, st);
  cudaMemsetAsync(v.dc + DC_ERR, 0, sizeof(int), st);
  AGB_LAUNCH(k_prep, nblocks(N), BLK, st, v);
  AGB_LAUNCH(k_pack_geom<R>, nblocks(N), BLK, st, v);
  AGB_LAUNCH(k_tile_box<R>, nblocks(32LL * ((N + 31) / 32)), BLK, st, v);
  nl += 3;
  stage_mark(s, 1);
  AGB_LAUNCH(k_cell_count, nblocks(N), BLK, st, v);
  agb_scan_excl(v.bucket_count, v.bucket_start, v.dc + DC_NB, v.dc + DC_C0 + 7, v.nbuckets, s->scan_scratch, st);
  AGB_LAUNCH(k_cell_fill, nblocks(N), BLK, st, v);
  if (v.skin > 0.0f) {
    /* candidates searched only when an atom has moved skin/2 (the search
       kernels return at once otherwise), filtered at every evaluation */
    cudaMemsetAsync(v.dc + DC_REBUILD, 0, sizeof(int), st);
    AGB_LAUNCH(k_skin_check, nblocks(N), BLK, st, v);
    AGB_LAUNCH(k_skin_len, 1, 32, st, v);
    AGB_LAUNCH(k_cand_count27, nblocks(27LL * N), BLK, st, v);
    agb_scan_excl(v.nl_c27, v.nl_o27, v.dc + DC_CLEN, v.dc + DC_CTOT, 27 * N, s->scan_scratch, st);
    AGB_LAUNCH(k_cand_emit27, nblocks(27LL * N), BLK, st, v);
    AGB_LAUNCH(k_cand_offsets, nblocks(N), BLK, st, v);
    AGB_LAUNCH(k_cand_flag, nblocks(s->cap_cand), BLK, st, v);
    agb_scan_excl(v.cand_flag, v.cand_scan, v.dc + DC_NCAND, v.dc + DC_NL, s->cap_cand, s->scan_scratch, st);
    AGB_LAUNCH(k_cand_nl_emit, nblocks(s->cap_cand), BLK, st, v);
    AGB_LAUNCH(k_cand_nl_offsets, nblocks(N), BLK, st, v);
    AGB_LAUNCH(k_nl_rank, nblocks(s->cap_nl), BLK, st, v);
    nl += 9 + 2 * AGB_SCAN_LAUNCHES;
  } else {
    cudaMemsetAsync(v.dc + DC_SLABMAX, 0, sizeof(int), st);
    if (v.nl_cells)
      AGB_LAUNCH(k_nl_cells, nblocks(27LL * N), BLK, st, v);
    else
      AGB_LAUNCH(k_nl_c27, nblocks(27LL * N), BLK, st, v);
    agb_scan_excl(v.nl_c27, v.nl_o27, v.dc + DC_N27, v.dc + DC_NL, 27 * N, s->scan_scratch, st);
    AGB_LAUNCH(k_nl_rank27, nblocks(32LL * N), BLK, st, v);
    nl += 2 + AGB_SCAN_LAUNCHES;
  }
  nl += 2 + AGB_SCAN_LAUNCHES; /* cell grid */
  stage_mark(s, 2);
  AGB_LAUNCH(k_l2_count<R>, nblocks(s->cap_nl), BLK, st, v);
  agb_scan_excl(v.lv_cnt[2], v.lv_off[2], v.dc + DC_NL, v.dc + DC_L0 + 2, s->cap_nl, s->scan_scratch, st);
  AGB_LAUNCH(k_l2_emit<R>, nblocks(s->cap_nl), BLK, st, v);
  nl += 2 + AGB_SCAN_LAUNCHES;
  for (int m = 3; m <= AGB_MAX_ORDER; m++) {
    int g = nblocks(v.cap[m - 1]);
    switch (m) {
      case 3: AGB_LAUNCH((k_lm_count<R, 3>), g, BLK, st, v); break;
      case 4: AGB_LAUNCH((k_lm_count<R, 4>), g, BLK, st, v); break;
      default: AGB_LAUNCH((k_lm_count<R, 5>), g, BLK, st, v); break;
    }
    /* the scan also maps each new record to its generating overlap */
    agb_scan_excl_owner(v.lv_cnt[m], v.lv_off[m], v.dc + DC_L0 + m - 1, v.dc + DC_L0 + m, v.cap[m - 1],
                        s->scan_scratch, st, v.lv_own[m], v.cap[m]);
    const int ge = nblocks(v.cap[m]);
    switch (m) {
      case 3: AGB_LAUNCH((k_lm_emit<R, 3>), ge, BLK, st, v); break;
      case 4: AGB_LAUNCH((k_lm_emit<R, 4>), ge, BLK, st, v); break;
      default: AGB_LAUNCH((k_lm_emit<R, 5>), ge, BLK, st, v); break;
    }
    nl += 2 + AGB_SCAN_LAUNCHES;
  }
  stage_mark(s, 3);
  AGB_LAUNCH(k_scaling, nblocks(N), BLK, st, v);
  AGB_LAUNCH(k_pack_sp<R>, nblocks(N), BLK, st, v);
  nl += 2;
  stage_mark(s, 4);
  /* the water-site stage needs only positions and spe (ready after the
     scaling factors) and writes only its own outputs, the HB gradient and
     derh: in a captured evaluation it runs on a side stream beside the pair
     stages and joins before the tree-derivative pass */
  if (side) {
    cudaEventRecord(s->fork_ev, st);
    cudaStreamWaitEvent(s->st2, s->fork_ev, 0);
    launch_ws<R>(s, v, s->st2);
    cudaEventRecord(s->join_ev, s->st2);
    nl += 4 + AGB_SCAN_LAUNCHES;
  }
  int dgrid = s->nitems < 148 * 32 ? s->nitems : 148 * 32; /* 64-thread descreening blocks */
  if (sizeof(R) == 4 && s->desc_smem > 0) {
    /* a block on every SM, of as many warps as the half items fill (the
       warps take them in turn from a counter: more warps than half items
       per SM would leave the later SMs without work) */
    const int units = 2 * s->nitems;
    int grid = units > 148 ? 148 : (units < 1 ? 1 : units);
    int nw = (units + 147) / 148;
    nw = nw > DS_WARPS ? DS_WARPS : (nw < 1 ? 1 : nw);
    k_descreen_s<<<grid, nw * 32, s->desc_smem, st>>>(v, s->items, s->nitems);
  } else {
    AGB_LAUNCH(k_descreen_t<R>, dgrid > 0 ? dgrid : 1, ITILE / 2, st, v, s->items, s->nitems, s->nch);
  }
  nl += 1;
  }
  const int pgrid = s->nitems < 148 * 16 ? (s->nitems > 0 ? s->nitems : 1) : 148 * 16;
  if (seg < 0) shard_allreduce(s, 0, st);
  if (seg < 0 || seg == 1) {
  AGB_LAUNCH(k_born<R>, nblocks(N), BLK, st, v);
  nl += 1;
  stage_mark(s, 5);
  if (s->tiled_pairs)
    AGB_LAUNCH(k_agb_t<R>, pgrid, ITILE, st, v, s->items, s->nitems, s->nch);
  else if (sizeof(R) == 4 && !s->scalar_pairs) {
    /* a block on every SM, of as many warps (up to 16) as the items fill */
    const int grid = s->n_agb > 148 ? 148 : (s->n_agb < 1 ? 1 : s->n_agb);
    int nw = (s->n_agb + 147) / 148;
    nw = nw > 16 ? 16 : (nw < 1 ? 1 : nw);
    AGB_LAUNCH(k_agb_x2, grid, nw * 32, st, v, s->items_agb, s->n_agb);
  }
  else
    AGB_LAUNCH(k_agb_sym<R>, sym_grid(s->n_agb), 128, st, v, s->items_agb, s->n_agb);
  nl += 1;
  }
  if (seg < 0) shard_allreduce(s, 1, st);
  if (seg < 0 || seg == 2) {
  AGB_LAUNCH(k_agb_post<R>, nblocks(N), BLK, st, v);
  nl += 1;
  stage_mark(s, 6);
  if (s->tiled_pairs)
    AGB_LAUNCH(k_gbders_t<R>, pgrid, ITILE, st, v, s->items, s->nitems, s->nch);
  else if (sizeof(R) == 4 && !s->scalar_pairs)
    launch_gbders_x2(s, st);
  else if (s->compat)
    AGB_LAUNCH((k_gbders_sym<R, true>), sym_grid(s->n_gbd), 128, st, v, s->items_gbd, s->n_gbd);
  else
    AGB_LAUNCH((k_gbders_sym<R, false>), sym_grid(s->n_gbd), 128, st, v, s->items_gbd, s->n_gbd);
  nl += 1;
  }
  if (seg < 0) shard_allreduce(s, 2, st);
  if (seg < 0 || seg == 3) {
  AGB_LAUNCH(k_gbders_post<R>, nblocks(N), BLK, st, v);
  nl += 1;
  stage_mark(s, 7);
  if (side) {
    cudaStreamWaitEvent(st, s->join_ev, 0);
  } else if (s->nws > 0) {
    launch_ws<R>(s, v, st);
    nl += 4 + AGB_SCAN_LAUNCHES;
  }
  stage_mark(s, 8);
  if (!s->timing && seg < 0) {
    /* the orders are independent (each reads its own records and adds to
       the gradients with atomics): orders 3 and 5 on the side stream beside
       2 and 4, which splits the records about evenly and fills the tails */
    cudaEventRecord(s->tfork_ev, st);
    cudaStreamWaitEvent(s->st2, s->tfork_ev, 0);
    AGB_LAUNCH((k_tree_ders<R, 3>), nblocks(v.cap[3]), BLK, s->st2, v);
    AGB_LAUNCH((k_tree_ders<R, 5>), nblocks(v.cap[5]), BLK, s->st2, v);
    cudaEventRecord(s->tjoin_ev, s->st2);
    AGB_LAUNCH((k_tree_ders<R, 2>), nblocks(v.cap[2]), BLK, st, v);
    AGB_LAUNCH((k_tree_ders<R, 4>), nblocks(v.cap[4]), BLK, st, v);
    cudaStreamWaitEvent(st, s->tjoin_ev, 0);
    nl += 4;
  } else {
    for (int m = 2; m <= AGB_MAX_ORDER; m++) {
      switch (m) {
        case 2: AGB_LAUNCH((k_tree_ders<R, 2>), nblocks(v.cap[m]), BLK, st, v); break;
        case 3: AGB_LAUNCH((k_tree_ders<R, 3>), nblocks(v.cap[m]), BLK, st, v); break;
        case 4: AGB_LAUNCH((k_tree_ders<R, 4>), nblocks(v.cap[m]), BLK, st, v); break;
        default: AGB_LAUNCH((k_tree_ders<R, 5>), nblocks(v.cap[m]), BLK, st, v); break;
      }
      nl += 1;
    }
  }
  stage_mark(s, 9);
  AGB_LAUNCH(k_final, nblocks(N), BLK, st, v);
  agb_segment_sum(v.eatom, N, 7, v.inst_begin, s->ninst, s->esum, st);
  if (s->nws > 0)
    agb_segment_sum(v.ews, 0, 1, v.ws_begin, s->ninst, s->ehb_inst, st);
  else
    cudaMemsetAsync(s->ehb_inst, 0, sizeof(double) * s->ninst, st);
  AGB_LAUNCH(k_energies, 1, 128, st, s->esum, s->ehb_inst, s->ninst, s->o_energy, v.dc);
  nl += 4;
  stage_mark(s, 10);
  }
  if (seg < 0) s->nlaunch = nl;
}

/* in-place sums over the ranks of stage k's partial sums, one NCCL group
   on the instance stream (captured with the rest of the evaluation) */
static void shard_allreduce(agb_dev *s, int k, cudaStream_t st) {
  if (!s->comm) return;
  double *p[5];
  size_t n[5];
  int m = shard_bufs(s, k, p, n);
  ncclResult_t r = g_nccl.GroupStart();
  for (int q = 0; q < m && r == ncclSuccess; q++)
    r = g_nccl.AllReduce(p[q], p[q], n[q], ncclFloat64, ncclSum, s->comm, st);
  ncclResult_t r2 = g_nccl.GroupEnd();
  if (r == ncclSuccess) r = r2;
  if (r != ncclSuccess && !s->nccl_err) s->nccl_err = (int)r;
}

static int run_once(agb_dev *s) {
  if (s->timing) {
    if (s->precision == AGB_PREC_FP64)
      launch_all<double>(s);
    else
      launch_all<float>(s);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->st));
    for (int k = 0; k < 10; k++) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, s->ev[k], s->ev[k + 1]);
      s->stage_ms[k] = ms;
    }
    return 0;
  }
  if (!s->graph_ok) {
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
    if (s->precision == AGB_PREC_FP64)
      launch_all<double>(s);
    else
      launch_all<float>(s);
    CK(cudaStreamEndCapture(s->st, &graph));
    CK(cudaGraphInstantiate(&s->gexec, graph, 0));
    cudaGraphDestroy(graph);
    s->graph_ok = 1;
  }
  CK(cudaGraphLaunch(s->gexec, s->st));
  return 0;
}

/* reads the device counters of the evaluation just issued on s->st:
   0 done, 1 a buffer overflowed (grown: evaluate again), -1 error */
static int finish_eval(agb_dev *s) {
  {
    int dc[DC_SIZE];
    CK(cudaMemcpyAsync(dc, s->v.dc, sizeof(dc), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    s->last_stats[0] = dc[DC_NL];
    for (int m = 2; m <= AGB_MAX_ORDER; m++) s->last_stats[m - 1] = dc[DC_L0 + m];
    s->last_stats[6] = s->nws;
    s->last_stats[7] = dc[DC_ERR];
    s->last_stats[8] = s->nlaunch;
    s->last_stats[9] = dc[DC_NBUILD];
    int err = dc[DC_ERR];
    if (err & (AGB_ERR_NL_CAP | AGB_ERR_TREE_CAP | AGB_ERR_WS_CAP | AGB_ERR_CAND_CAP)) {
      /* grow what overflowed and evaluate again */
      if (dc[DC_NL] > s->cap_nl) s->cap_nl = 2 * dc[DC_NL];
      if (dc[DC_SLABMAX] > s->slab_w) s->slab_w = dc[DC_SLABMAX] + 4;
      if ((err & AGB_ERR_CAND_CAP) && dc[DC_CTOT] > s->cap_cand) s->cap_cand = 2 * dc[DC_CTOT];
      if (dc[DC_WSC] > s->cap_wsc) s->cap_wsc = 2 * dc[DC_WSC];
      for (int m = 2; m <= AGB_MAX_ORDER; m++)
        if (dc[DC_L0 + m] > s->cap[m]) s->cap[m] = 2 * dc[DC_L0 + m];
      if (s->graph_ok) {
        cudaGraphExecDestroy(s->gexec);
        s->graph_ok = 0;
      }
      tree_free(s);
      if (tree_alloc(s)) return -1;
      return 1;
    }
    if (err & AGB_ERR_NONFINITE) FAIL("non-finite energy");
    return 0;
  }
}

extern "C" int agb_dev_evaluate(agb_dev *s) {
  CK(cudaSetDevice(s->device));
  if (!s->order_ok && order_pair_slots(s)) return -1;
  /* each attempt can reveal the overflow of one more buffer (a level's
     size is only known once the level below fits) */
  for (int attempt = 0; attempt < 16; attempt++) {
    if (run_once(s)) return -1;
    if (s->nccl_err) {
      int e = s->nccl_err;
      s->nccl_err = 0;
      FAIL("NCCL all-reduce of the sharded pair sums: %s", g_nccl.GetErrorString((ncclResult_t)e));
    }
    const int r = finish_eval(s);
    if (r <= 0) return r;
  }
  FAIL("overlap buffers did not converge after regrowing");
}

/* several independent evaluations at once: every one whose captured graph
   is ready is launched on its own stream before any is waited for, so the
   latency-bound stages of one overlap the pair passes of another; each is
   then checked as agb_dev_evaluate checks it, and one whose buffers
   overflowed is grown and evaluated again on its own.  Evaluations that are
   not ready for a graph replay (first call, stage timing, sharded) are
   evaluated one after the other. */
extern "C" int agb_dev_evaluate_many(agb_dev *const *ss, int n) {
  int ready[64];
  if (n < 0 || n > 64) FAIL("%d evaluations at once (at most 64)", n);
  for (int k = 0; k < n; k++) {
    agb_dev *s = ss[k];
    ready[k] = s->graph_ok && s->order_ok && !s->timing && !s->comm && s->shard_n <= 1;
    if (!ready[k] && agb_dev_evaluate(s)) return -1;
  }
  for (int k = 0; k < n; k++)
    if (ready[k]) {
      CK(cudaSetDevice(ss[k]->device));
      CK(cudaGraphLaunch(ss[k]->gexec, ss[k]->st));
    }
  for (int k = 0; k < n; k++)
    if (ready[k]) {
      CK(cudaSetDevice(ss[k]->device));
      const int r = finish_eval(ss[k]);
      if (r < 0) return -1;
      if (r == 1 && agb_dev_evaluate(ss[k])) return -1;
    }
  return 0;
}

extern "C" int agb_dev_shard_unique_id(void *id, int nbytes) {
  if (nbytes < (int)sizeof(ncclUniqueId)) FAIL("unique id buffer of %d bytes, need %d", nbytes, (int)sizeof(ncclUniqueId));
  if (nccl_load()) return -1;
  ncclUniqueId u;
  ncclResult_t r = g_nccl.GetUniqueId(&u);
  if (r != ncclSuccess) FAIL("ncclGetUniqueId: %s", g_nccl.GetErrorString(r));
  memcpy(id, &u, sizeof(u));
  return (int)sizeof(u);
}

/* this instance as rank `rank` of `nranks`: pair-stage items split over the
   ranks; with `id` (the same ncclUniqueId on every rank) the partial sums
   are added over the ranks by NCCL inside each evaluation, without it the
   evaluation only runs segment by segment (agb_dev_shard_segment) and the
   caller adds them.  nranks = 1 without id undoes the sharding. */
extern "C" int agb_dev_shard(agb_dev *s, int rank, int nranks, const void *id, int nbytes) {
  CK(cudaSetDevice(s->device));
  if (nranks < 1 || rank < 0 || rank >= nranks) FAIL("rank %d of %d", rank, nranks);
  CK(cudaStreamSynchronize(s->st));
  if (s->graph_ok) {
    cudaGraphExecDestroy(s->gexec);
    s->graph_ok = 0;
  }
  if (s->comm) {
    g_nccl.CommDestroy(s->comm);
    s->comm = NULL;
  }
  if (id) {
    if (nbytes < (int)sizeof(ncclUniqueId)) FAIL("unique id of %d bytes, need %d", nbytes, (int)sizeof(ncclUniqueId));
    if (nccl_load()) return -1;
    ncclUniqueId u;
    memcpy(&u, id, sizeof(u));
    ncclComm_t c;
    ncclResult_t r = g_nccl.CommInitRank(&c, nranks, u, rank);
    if (r != ncclSuccess) FAIL("ncclCommInitRank(rank %d of %d): %s", rank, nranks, g_nccl.GetErrorString(r));
    s->comm = c;
  }
  s->shard_rank = rank;
  s->shard_n = nranks;
  return build_items(s, s->nch, s->jb);
}

/* one segment of a sharded evaluation without a communicator, launched
   directly and waited for: 0 .. 3, with the partial sums of pair stage k
   exchanged through agb_dev_shard_buffers between segments k and k+1 */
extern "C" int agb_dev_shard_segment(agb_dev *s, int k) {
  CK(cudaSetDevice(s->device));
  if (k < 0 || k > 3) FAIL("segment %d", k);
  if (s->comm) FAIL("segments are for sharding without a communicator");
  if (k == 0 && !s->order_ok && order_pair_slots(s)) return -1;
  if (s->precision == AGB_PREC_FP64)
    launch_all<double>(s, k);
  else
    launch_all<float>(s, k);
  CK(cudaGetLastError());
  int dc[DC_SIZE];
  CK(cudaMemcpyAsync(dc, s->v.dc, sizeof(dc), cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  if (dc[DC_ERR] & (AGB_ERR_NL_CAP | AGB_ERR_TREE_CAP | AGB_ERR_WS_CAP | AGB_ERR_CAND_CAP))
    FAIL("buffer overflow in a segmented evaluation (error word %d): evaluate once unsharded first", dc[DC_ERR]);
  if (k == 3) {
    s->last_stats[0] = dc[DC_NL];
    for (int m = 2; m <= AGB_MAX_ORDER; m++) s->last_stats[m - 1] = dc[DC_L0 + m];
    s->last_stats[7] = dc[DC_ERR];
    if (dc[DC_ERR] & AGB_ERR_NONFINITE) FAIL("non-finite energy");
  }
  return 0;
}

/* stage k's partial sums to (store 0) or from (store 1) host memory,
   concatenated; returns the element count (host may be NULL to ask) */
extern "C" long long agb_dev_shard_buffers(agb_dev *s, int k, double *host, int store) {
  CK(cudaSetDevice(s->device));
  if (k < 0 || k > 2) FAIL("stage %d", k);
  double *p[5];
  size_t n[5], tot = 0;
  int m = shard_bufs(s, k, p, n);
  for (int q = 0; q < m; q++) {
    if (host) {
      if (store)
        CK(cudaMemcpy(p[q], host + tot, sizeof(double) * n[q], cudaMemcpyHostToDevice));
      else
        CK(cudaMemcpy(host + tot, p[q], sizeof(double) * n[q], cudaMemcpyDeviceToHost));
    }
    tot += n[q];
  }
  return (long long)tot;
}

extern "C" int agb_dev_download(agb_dev *s, double *energies, double *sp, double *br, double *surf_area,
                                double *dgbdr, double *dvwdr, double *decav, double *dehb) {
  CK(cudaSetDevice(s->device));
  size_t n = sizeof(double) * s->natoms;
  View &v = s->v;
  if (energies) CK(cudaMemcpyAsync(energies, s->o_energy, sizeof(double) * 7 * s->ninst, cudaMemcpyDeviceToHost, s->st));
  if (sp) CK(cudaMemcpyAsync(sp, v.o_sp, n, cudaMemcpyDeviceToHost, s->st));
  if (br) CK(cudaMemcpyAsync(br, v.o_br, n, cudaMemcpyDeviceToHost, s->st));
  if (surf_area) CK(cudaMemcpyAsync(surf_area, v.o_sa, n, cudaMemcpyDeviceToHost, s->st));
  if (dgbdr) CK(cudaMemcpyAsync(dgbdr, v.o_gb, 3 * n, cudaMemcpyDeviceToHost, s->st));
  if (dvwdr) CK(cudaMemcpyAsync(dvwdr, v.o_gv, 3 * n, cudaMemcpyDeviceToHost, s->st));
  if (decav) CK(cudaMemcpyAsync(decav, v.o_gc, 3 * n, cudaMemcpyDeviceToHost, s->st));
  if (dehb) CK(cudaMemcpyAsync(dehb, v.o_gh, 3 * n, cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  return 0;
}

/* device-array variants: the instance stream first waits for the work
   already queued on the caller's stream; after the output copies the
   caller's stream waits for the instance stream */
extern "C" int agb_dev_upload_coords_dev(agb_dev *s, const double *x, const double *y, const double *z,
                                         void *stream) {
  CK(cudaSetDevice(s->device));
  CK(cudaEventRecord(s->xev, (cudaStream_t)stream));
  CK(cudaStreamWaitEvent(s->st, s->xev, 0));
  size_t b = sizeof(double) * s->natoms;
  CK(cudaMemcpyAsync((void *)s->v.x_ext, x, b, cudaMemcpyDeviceToDevice, s->st));
  CK(cudaMemcpyAsync((void *)s->v.y_ext, y, b, cudaMemcpyDeviceToDevice, s->st));
  CK(cudaMemcpyAsync((void *)s->v.z_ext, z, b, cudaMemcpyDeviceToDevice, s->st));
  return 0;
}

extern "C" int agb_dev_download_dev(agb_dev *s, double *energies, double *sp, double *br, double *surf_area,
                                    double *dgbdr, double *dvwdr, double *decav, double *dehb, void *stream) {
  CK(cudaSetDevice(s->device));
  size_t n = sizeof(double) * s->natoms;
  View &v = s->v;
  const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
  if (energies) CK(cudaMemcpyAsync(energies, s->o_energy, sizeof(double) * 7 * s->ninst, k, s->st));
  if (sp) CK(cudaMemcpyAsync(sp, v.o_sp, n, k, s->st));
  if (br) CK(cudaMemcpyAsync(br, v.o_br, n, k, s->st));
  if (surf_area) CK(cudaMemcpyAsync(surf_area, v.o_sa, n, k, s->st));
  if (dgbdr) CK(cudaMemcpyAsync(dgbdr, v.o_gb, 3 * n, k, s->st));
  if (dvwdr) CK(cudaMemcpyAsync(dvwdr, v.o_gv, 3 * n, k, s->st));
  if (decav) CK(cudaMemcpyAsync(decav, v.o_gc, 3 * n, k, s->st));
  if (dehb) CK(cudaMemcpyAsync(dehb, v.o_gh, 3 * n, k, s->st));
  CK(cudaEventRecord(s->xev, s->st));
  CK(cudaStreamWaitEvent((cudaStream_t)stream, s->xev, 0));
  return 0;
}

extern "C" void *agb_dev_stream(agb_dev *s) { return (void *)s->st; }

extern "C" int agb_dev_set_timing(agb_dev *s, int enable) {
  s->timing = enable != 0;
  return 0;
}

extern "C" int agb_dev_stage_times(agb_dev *s, double *ms, int n) {
  int k;
  for (k = 0; k < n && k < 10; k++) ms[k] = s->stage_ms[k];
  return 10;
}

extern "C" int agb_dev_stats(agb_dev *s, long long *out, int n) {
  for (int k = 0; k < n && k < 16; k++) out[k] = s->last_stats[k];
  return 10;
}

/* debug fetch ids */
enum {
  DBG_NL_COUNT = 0, /* int[natoms] */
  DBG_NL_LIST,      /* int[nl] */
  DBG_LEVEL_PAR,    /* + m*16: int[m][cap] order-m parents (first n rows valid) */
  DBG_ATOM = 100,   /* + k: double[natoms] per-atom array k */
  DBG_WS_SP = 200,  /* double[nws] */
  DBG_WS_POS,       /* double[3*nws] */
  DBG_SLOT_ATOM,    /* int[natoms]: the atom in each pair slot */
};

extern "C" long long agb_dev_debug_fetch(agb_dev *s, int what, void *out, long long cap) {
  cudaSetDevice(s->device);
  cudaStreamSynchronize(s->st);
  View &v = s->v;
  int N = s->natoms;
  if (what == DBG_NL_COUNT) {
    if (cap < N) return -1;
    cudaMemcpy(out, v.nl_count, sizeof(int) * N, cudaMemcpyDeviceToHost);
    return N;
  }
  if (what == DBG_NL_LIST) {
    long long n = s->last_stats[0];
    if (n > cap) return -n;
    cudaMemcpy(out, v.nl_list, sizeof(int) * n, cudaMemcpyDeviceToHost);
    return n;
  }
  if (what >= DBG_LEVEL_PAR && what < DBG_LEVEL_PAR + 16 * (AGB_MAX_ORDER + 1) && (what - DBG_LEVEL_PAR) % 16 == 0) {
    int m = (what - DBG_LEVEL_PAR) / 16;
    if (m < 2 || m > AGB_MAX_ORDER) return -1;
    long long n = s->last_stats[m - 1];
    if ((long long)m * n > cap) return -(long long)m * n;
    int *o = (int *)out;
    for (int k = 0; k < m; k++) cudaMemcpy(o + k * n, v.par[m] + (size_t)k * s->cap[m], sizeof(int) * n, cudaMemcpyDeviceToHost);
    return n;
  }
  if (what >= DBG_ATOM && what < DBG_ATOM + 32) {
    double *arrs[] = {v.volumep, v.surf, v.surf_f, v.sp, v.spe, v.psvol, v.gammap, v.bfil, v.bder, v.br, v.brw,
                      v.dera, v.q2ab, v.abrw, v.deru, v.derv, v.derh, v.derus, v.dervs, v.acc_beta};
    int k = what - DBG_ATOM;
    if (k >= (int)(sizeof(arrs) / sizeof(arrs[0])) || cap < N) return -1;
    cudaMemcpy(out, arrs[k], sizeof(double) * N, cudaMemcpyDeviceToHost);
    return N;
  }
  if (what == DBG_SLOT_ATOM) {
    if (cap < N) return -1;
    cudaMemcpy(out, v.slot_atom, sizeof(int) * N, cudaMemcpyDeviceToHost);
    return N;
  }
  if (what == DBG_WS_SP) {
    if (cap < s->nws) return -1;
    if (s->nws) cudaMemcpy(out, v.wsp, sizeof(double) * s->nws, cudaMemcpyDeviceToHost);
    return s->nws;
  }
  if (what == DBG_WS_POS) {
    if (cap < 3LL * s->nws) return -1;
    if (s->nws == 0) return 0;
    if (s->precision == AGB_PREC_FP64) {
      cudaMemcpy(out, v.wpos, sizeof(double) * 3 * s->nws, cudaMemcpyDeviceToHost);
    } else {
      float *tmp = (float *)malloc(sizeof(float) * 3 * s->nws);
      cudaMemcpy(tmp, v.wpos, sizeof(float) * 3 * s->nws, cudaMemcpyDeviceToHost);
      for (int k = 0; k < 3 * s->nws; k++) ((double *)out)[k] = tmp[k];
      free(tmp);
    }
    return s->nws;
  }
  return -1;
}

/* Autotuner for the pair-stage decomposition: tries partner-chunk counts
   for the one-sided descreening pass and j-run lengths for the symmetric
   passes on the current coordinates (stage timers, median of `reps`
   evaluations after one warm-up), keeps the fastest and returns
   params = {nch, jb, invb_us, agb_gbders_us}.  With params_in set, applies
   them without timing. */
extern "C" int agb_dev_autotune(agb_dev *s, int reps, const int *params_in, int *params_out) {
  CK(cudaSetDevice(s->device));
  if (params_in) {
    if (build_items(s, params_in[0], params_in[1])) return -1;
    if (params_out) {
      params_out[0] = s->nch;
      params_out[1] = s->jb;
      params_out[2] = params_out[3] = -1;
    }
    return 0;
  }
  /* timings differ between GPUs, and ranks whose work lists differ would
     split the pairs inconsistently */
  if (s->shard_n > 1) FAIL("a sharded instance is not tuned: pass the same explicit parameters on every rank");
  if (reps < 1) reps = 1;
  int timing = s->timing;
  s->timing = 1;
  int maxh = 1;
  for (int I = 0; I < s->ninst; I++)
    if (s->h_inst_nheavy[I] > maxh) maxh = s->h_inst_nheavy[I];
  const int nchs[] = {1, 2, 3, 4, 6, 8, 12, 16, 24, 32};
  const int jbs[] = {2, 4, 8, 16, 32};
  double best = 1e30;
  int bn = 1, bj = s->jb;
  double samp[16];
  for (size_t a = 0; a < sizeof(nchs) / sizeof(nchs[0]); a++) {
    if (nchs[a] > 1 && maxh / nchs[a] < 128) break;
    if (build_items(s, nchs[a], bj)) return -1;
    for (int r = 0; r <= reps; r++) {
      if (agb_dev_evaluate(s)) return -1;
      if (r) samp[r - 1] = s->stage_ms[4];
    }
    double m = samp[0];
    for (int r = 1; r < reps; r++) m = samp[r] < m ? samp[r] : m;
    if (m < best) {
      best = m;
      bn = nchs[a];
    }
  }
  double tinvb = best;
  best = 1e30;
  for (size_t a = 0; a < sizeof(jbs) / sizeof(jbs[0]); a++) {
    if (build_items(s, bn, jbs[a])) return -1;
    for (int r = 0; r <= reps; r++) {
      if (agb_dev_evaluate(s)) return -1;
      if (r) samp[r - 1] = s->stage_ms[5] + s->stage_ms[6];
    }
    double m = samp[0];
    for (int r = 1; r < reps; r++) m = samp[r] < m ? samp[r] : m;
    if (m < best) {
      best = m;
      bj = jbs[a];
    }
  }
  if (build_items(s, bn, bj)) return -1;
  s->timing = timing;
  if (params_out) {
    params_out[0] = bn;
    params_out[1] = bj;
    params_out[2] = (int)(1e3 * tinvb);
    params_out[3] = (int)(1e3 * best);
  }
  return 0;
}


/* ------------------------------------------------------------------------ */
/* learned surrogate: radial neighbour features per atom                    */
/* ------------------------------------------------------------------------ */
#define SF_NC 5              /* atom classes (C, N, O, S, H by radius) */
#define SF_NB 32             /* radial basis functions per class */
#define SF_NF (SF_NC * SF_NB) /* features per atom */
#define SF_RC 8.0f           /* cutoff (A) */
#define SF_W 4               /* basis functions each side of the nearest centre */

/* the class of every atom: the class radius within 1e-3 A of its radius */
__global__ void k_set_class(View v, int nc, float r0, float r1, float r2, float r3, float r4, int *unmatched) {
  AGB_GRID_STRIDE(g, v.natoms) {
    const float cr[SF_NC] = {r0, r1, r2, r3, r4};
    float r = (float)(v.r[g] - C_RINC);
    int c = -1;
    for (int k = 0; k < nc && k < SF_NC; k++)
      if (fabsf(r - cr[k]) < 1e-3f) c = k;
    v.sclass[g] = (signed char)c;
    if (c < 0) atomicAdd(unmatched, 1);
  }
}

/* the surrogate's grid: bucket of every atom (cell edge SF_RC) */
__device__ __forceinline__ int sf_key(int cx, int cy, int cz) {
  return (cx & 1023) | ((cy & 1023) << 10) | ((cz & 1023) << 20);
}

__global__ void k_sf_cell_count(View v) {
  AGB_GRID_STRIDE(g, v.natoms) {
    int I = v.inst_of[g];
    f4 p = v.pos[g];
    int cx, cy, cz;
    cell_of(p.x, p.y, p.z, 1.0f / SF_RC, cx, cy, cz);
    int b = v.sf_bbegin[I] + cell_hash(cx, cy, cz, v.sf_bmask[I]);
    v.sf_abucket[g] = b;
    atomicAdd(&v.sf_bcount[b], 1);
  }
}

__global__ void k_sf_cell_fill(View v) {
  AGB_GRID_STRIDE(g, v.natoms) {
    f4 p = v.pos[g];
    int cx, cy, cz;
    cell_of(p.x, p.y, p.z, 1.0f / SF_RC, cx, cy, cz);
    int b = v.sf_abucket[g];
    int slot = v.sf_bstart[b] + atomicAdd(&v.sf_bcursor[b], 1);
    p.w = (float)v.sclass[g];
    v.sf_spos[slot] = p;
    v.sf_sid[slot] = make_int2((int)g, sf_key(cx, cy, cz));
  }
}

/* one neighbour at distance d < SF_RC into a feature row (class c):
   Gaussians of width equal to their spacing, centres k * SF_RC / (SF_NB-1),
   times a cosine cutoff; basis functions beyond SF_W spacings of d are not
   added (they are below e^-8 of the nearest) */
__device__ __forceinline__ void sf_add(float *row, int c, float d) {
  const float delta = SF_RC / (SF_NB - 1), inv2s2 = 0.5f / (delta * delta);
  const float fc = 0.5f * (__cosf(3.14159265358979f * d / SF_RC) + 1.f);
  const int kc = __float2int_rn(d / delta);
  const int k0 = max(0, kc - SF_W), k1 = min(SF_NB - 1, kc + SF_W);
  for (int k = k0; k <= k1; k++) {
    float u = d - (float)k * delta;
    row[c * SF_NB + k] += fc * __expf(-u * u * inv2s2);
  }
}

/* sf_add into a row shared by the lanes of a warp (shared-memory atomics) */
__device__ __forceinline__ void sf_add_shared(float *row, int c, float d) {
  const float delta = SF_RC / (SF_NB - 1), inv2s2 = 0.5f / (delta * delta);
  const float fc = 0.5f * (__cosf(3.14159265358979f * d / SF_RC) + 1.f);
  const int kc = __float2int_rn(d / delta);
  const int k0 = max(0, kc - SF_W), k1 = min(SF_NB - 1, kc + SF_W);
  for (int k = k0; k <= k1; k++) {
    float u = d - (float)k * delta;
    atomicAdd(&row[c * SF_NB + k], fc * __expf(-u * u * inv2s2));
  }
}

/* features of every atom: for each neighbour class, the basis sum over the
   atoms of that class within SF_RC, plus the atom's own class at d = 0.  One
   warp per atom.  Its lanes test the slots of the 27 grid cells around the
   atom 32 at a time and append the neighbours within SF_RC (distance,
   class) to a per-warp list in shared memory; every time the list holds 32,
   each lane takes one and adds its basis terms to the warp's row of sums
   (shared-memory atomics), so the basis work runs on full warps whatever
   the share of candidates in range (about 1 in 6).  Output: bf16
   [natoms][SF_NF], internal order, each feature (x - mean) * invstd when
   mean / invstd are given. */
#define SF_WARPS 4
__global__ void __launch_bounds__(32 * SF_WARPS) k_sfeat(View v, const float *__restrict__ mean,
                                                         const float *__restrict__ invstd,
                                                         __nv_bfloat16 *__restrict__ out) {
  __shared__ float srow[SF_WARPS][SF_NF];
  __shared__ float sdist[SF_WARPS][64];
  __shared__ int scls[SF_WARPS][64];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  float *row = srow[wp];
  float *bd = sdist[wp];
  int *bc = scls[wp];
  const float rc2 = SF_RC * SF_RC;
  const long long nw = (long long)gridDim.x * SF_WARPS;
  for (long long gg = (long long)blockIdx.x * SF_WARPS + wp; gg < v.natoms; gg += nw) {
    const int g = (int)gg;
    for (int f = lane; f < SF_NF; f += 32) row[f] = 0.f;
    __syncwarp();
    const int I = v.inst_of[g];
    const f4 pi = v.pos[g];
    const int ci = v.sclass[g];
    if (lane == 0 && ci >= 0) sf_add_shared(row, ci, 0.f);
    int cx, cy, cz;
    cell_of(pi.x, pi.y, pi.z, 1.0f / SF_RC, cx, cy, cz);
    int nbuf = 0; /* warp-uniform */
    for (int c = 0; c < 27; c++) {
      const int ax = cx + c % 3 - 1, ay = cy + (c / 3) % 3 - 1, az = cz + c / 9 - 1;
      const int b = v.sf_bbegin[I] + cell_hash(ax, ay, az, v.sf_bmask[I]);
      const int key = sf_key(ax, ay, az);
      const int s0 = v.sf_bstart[b], s1 = s0 + v.sf_bcount[b];
      for (int q0 = s0; q0 < s1; q0 += 32) {
        const int q = q0 + lane;
        bool in = false;
        float d = 0.f;
        int cj = 0;
        if (q < s1) {
          const int2 id = v.sf_sid[q];
          const f4 pj = v.sf_spos[q];
          if (id.y == key && id.x != g && pj.w >= 0.f) {
            const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
            const float d2 = dx * dx + dy * dy + dz * dz;
            if (d2 < rc2) {
              in = true;
              d = sqrtf(d2);
              cj = (int)pj.w;
            }
          }
        }
        const unsigned m = __ballot_sync(0xffffffffu, in);
        if (in) {
          const int pos = nbuf + __popc(m & ((1u << lane) - 1u));
          bd[pos] = d;
          bc[pos] = cj;
        }
        nbuf += __popc(m); /* at most 63 */
        if (nbuf >= 32) {
          __syncwarp();
          sf_add_shared(row, bc[lane], bd[lane]);
          __syncwarp();
          if (lane < nbuf - 32) { /* the rest to the front (read 32 + lane, write lane) */
            bd[lane] = bd[32 + lane];
            bc[lane] = bc[32 + lane];
          }
          __syncwarp();
          nbuf -= 32;
        }
      }
    }
    __syncwarp();
    if (lane < nbuf) sf_add_shared(row, bc[lane], bd[lane]);
    __syncwarp();
    for (int f = lane; f < SF_NF; f += 32) {
      float x = row[f];
      if (mean) x = (x - mean[f]) * invstd[f];
      out[(size_t)g * SF_NF + f] = __float2bfloat16(x);
    }
    __syncwarp(); /* the row is read before the next atom clears it */
  }
}

extern "C" int agb_dev_surrogate_classes(agb_dev *s, const double *class_radii, int nc, int *unmatched) {
  if (nc < 1 || nc > SF_NC) FAIL("surrogate: 1 to %d atom classes, not %d", SF_NC, nc);
  CK(cudaSetDevice(s->device));
  float r[SF_NC] = {-1.f, -1.f, -1.f, -1.f, -1.f};
  for (int k = 0; k < nc; k++) r[k] = (float)class_radii[k];
  int *cnt;
  CK(cudaMalloc((void **)&cnt, sizeof(int)));
  CK(cudaMemsetAsync(cnt, 0, sizeof(int), s->st));
  k_set_class<<<nblocks(s->natoms), BLK, 0, s->st>>>(s->v, nc, r[0], r[1], r[2], r[3], r[4], cnt);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(unmatched, cnt, sizeof(int), cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  cudaFree(cnt);
  return 0;
}

/* features of the coordinates of the last evaluation (internal order),
   queued on the instance stream (which agbnp3_stream returns) */
extern "C" int agb_dev_surrogate_features(agb_dev *s, const float *mean, const float *invstd, void *out) {
  CK(cudaSetDevice(s->device));
  View &v = s->v;
  CK(cudaMemsetAsync(v.sf_bcount, 0, sizeof(int) * v.sf_nbuckets, s->st));
  CK(cudaMemsetAsync(v.sf_bcursor, 0, sizeof(int) * v.sf_nbuckets, s->st));
  k_sf_cell_count<<<nblocks(s->natoms), BLK, 0, s->st>>>(v);
  agb_scan_excl(v.sf_bcount, v.sf_bstart, v.sf_dc, v.sf_dc + 1, v.sf_nbuckets, s->scan_scratch, s->st);
  k_sf_cell_fill<<<nblocks(s->natoms), BLK, 0, s->st>>>(v);
  int grid = (s->natoms + SF_WARPS - 1) / SF_WARPS;
  if (grid > 148 * 16) grid = 148 * 16;
  k_sfeat<<<grid, 32 * SF_WARPS, 0, s->st>>>(v, mean, invstd, (__nv_bfloat16 *)out);
  CK(cudaGetLastError());
  return 0;
}
