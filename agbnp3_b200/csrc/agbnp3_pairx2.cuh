/*
 * FP32 pair passes in packed two-lane arithmetic (sm_100 f32x2: one
 * FFMA2/FADD2/FMUL2 instruction does the same operation on both halves of
 * a float2).  The pair passes are bound by instruction issue, not by the
 * FMA pipe: measured on B200, FFMA2 runs at the scalar FFMA flop rate
 * (73.7 vs 71.7 TFLOP/s) but leaves every other issue slot free, so with
 * one integer instruction interleaved per FFMA2 the FMA rate stays at
 * 65 TFLOP/s where scalar code falls to 51.  Here each packed operation
 * evaluates two pairs at once: a lane's i atoms are held in packed pairs
 * (one atom in each half), the j atom's operands are broadcast to both
 * halves from shared memory, where the j tile is stored with every value
 * duplicated.
 *
 * Included by agbnp3_dev.cu (uses its View, operand arrays and helpers).
 */
#pragma once

__device__ __forceinline__ float2 x2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 ex2_2(float2 a) {
  return make_float2(GbExp<float>::ex(a.x), GbExp<float>::ex(a.y));
}
__device__ __forceinline__ float2 rsqrt_2(float2 a) { return make_float2(p_rsqrt(a.x), p_rsqrt(a.y)); }
__device__ __forceinline__ float2 rot1_2(float2 a) { return make_float2(rot1(a.x), rot1(a.y)); }
__device__ __forceinline__ float fold(float2 a) { return a.x + a.y; }
__device__ __forceinline__ float lo_hi(float2 a, int h) { return h ? a.y : a.x; }

/* ------------------------------------------------------------------------ */
/* GB pair energy, constant-B gradient and A_i (agbnp3_cpu_simd_kernels.c:  */
/* 66-151, 329-460), the symmetric decomposition of k_agb_sym: a warp owns  */
/* an i block of 2 * AX_NP 32-atom tiles (lane l keeps atoms I+l, I+32+l,   */
/* ..., packed two per float2: tiles 2p and 2p+1 in pair p) and walks a run */
/* of 32-atom j tiles.  The j tile sits in shared memory, each value twice  */
/* ((x,x,y,y), (z,z,q,q), (B,B,1/B,1/B)); in rotation step r lane l reads   */
/* j atom (l + r) mod 32 and adds its pairs with its 2 * AX_NP i atoms to    */
/* the j atom's sums, which travel to lane l - 1 for the next step, so      */
/* every unordered pair is evaluated once.                                  */
/* ------------------------------------------------------------------------ */
#define AX_NP 2
static_assert(SymNI<float>::agb == 2 * AX_NP, "the FP32 GB pair items hold i blocks of 2 * AX_NP tiles");

struct AxI {
  int i0;                                                               /* the lane's atom in the first i tile */
  float2 nx[AX_NP], ny[AX_NP], nz[AX_NP], q[AX_NP], b[AX_NP], c[AX_NP]; /* nx = -x */
};
struct AxP {
  float2 e[AX_NP], gx[AX_NP], gy[AX_NP], gz[AX_NP], at[AX_NP];
};
struct AxJ { /* sums of the j atom a lane holds, one partial per half */
  float2 gx, gy, gz, at;
};

/* one j tile.  FULL: every j atom valid and after the i block (no index
   tests); coincident atoms (d^2 = 0, contributing nothing, as in the
   reference's scalar kernel, agbnp3_cpu_simd_kernels.c:107-108) are then
   caught by a warp vote on the product of the step's d^2 values */
template <bool FULL>
__device__ __forceinline__ void agb_tile_x2(const AxI &I, AxP &P, AxJ &J, const float4 (*sj)[32], int lane, int j0,
                                            int a1) {
#pragma unroll 1
  for (int r = 0; r < 32; r++) {
    const int jj = (lane + r) & 31;
    const float4 A = sj[0][jj], B = sj[1][jj], C = sj[2][jj];
    const float2 jx = make_float2(A.x, A.y), jy = make_float2(A.z, A.w), jz = make_float2(B.x, B.y);
    const float2 jq = make_float2(B.z, B.w), jb = make_float2(C.x, C.y), jbi = make_float2(C.z, C.w);
    float2 dx[AX_NP], dy[AX_NP], dz[AX_NP], d2[AX_NP];
#pragma unroll
    for (int p = 0; p < AX_NP; p++) {
      dx[p] = add2(jx, I.nx[p]);
      dy[p] = add2(jy, I.ny[p]);
      dz[p] = add2(jz, I.nz[p]);
      d2[p] = fma2(dz[p], dz[p], fma2(dy[p], dy[p], mul2(dx[p], dx[p])));
    }
    bool mask;
    if (FULL) {
      float2 m = d2[0];
#pragma unroll
      for (int p = 1; p < AX_NP; p++) m = mul2(m, d2[p]);
      mask = __any_sync(FULLMASK, m.x * m.y == 0.f);
    } else {
      mask = true;
    }
    const int jr = j0 + jj;
#pragma unroll
    for (int p = 0; p < AX_NP; p++) {
      const float2 bb = mul2(I.b[p], jb);
      const float2 et = ex2_2(mul2(mul2(I.c[p], jbi), d2[p]));
      float2 f = rsqrt_2(fma2(bb, et, d2[p]));
      if (mask) { /* rare (FULL) or boundary tiles: per-pair validity */
        const int i0 = I.i0 + 64 * p, i1 = i0 + 32; /* atoms of the pair's halves (valid if < a1) */
        const bool v0 = d2[p].x > 0.f && (FULL || (jr < a1 && i0 < jr));
        const bool v1 = d2[p].y > 0.f && (FULL || (jr < a1 && i1 < jr));
        f.x = v0 ? f.x : 0.f;
        f.y = v1 ? f.y : 0.f;
      }
      const float2 qf = mul2(mul2(I.q[p], jq), f);
      P.e[p] = add2(P.e[p], qf);
      const float2 qf3 = mul2(qf, mul2(f, f));
      const float2 eq = mul2(et, qf3);
      const float2 mw = fma2(eq, x2(-0.25f), qf3);
      P.gx[p] = fma2(mw, dx[p], P.gx[p]);
      P.gy[p] = fma2(mw, dy[p], P.gy[p]);
      P.gz[p] = fma2(mw, dz[p], P.gz[p]);
      J.gx = fma2(mw, dx[p], J.gx); /* the j side takes -mw d: negated when folded */
      J.gy = fma2(mw, dy[p], J.gy);
      J.gz = fma2(mw, dz[p], J.gz);
      const float2 at = mul2(eq, fma2(d2[p], x2(0.25f), bb));
      P.at[p] = add2(P.at[p], at);
      J.at = add2(J.at, at);
    }
    J.gx = rot1_2(J.gx);
    J.gy = rot1_2(J.gy);
    J.gz = rot1_2(J.gz);
    J.at = rot1_2(J.at);
  }
}

/* 115 registers, one block of up to 16 warps per SM, whose warps take the
   items from a device counter (spread over the list by take_unit): 2-6 %
   faster than four 4-warp blocks per SM taking items in grid order (five
   such blocks, at 96 registers with spills, measured 2 % slower still) */
__global__ void __launch_bounds__(512, 1) k_agb_x2(View v, const int4 *__restrict__ items, int nitems) {
  __shared__ float4 sjt[16][3][32];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const float *X = pa<float>(v, PA_X), *Y = pa<float>(v, PA_Y), *Z = pa<float>(v, PA_Z);
  const float *Q = pa<float>(v, PA_Q), *Bv = pa<float>(v, PA_B), *BI = pa<float>(v, PA_BINV);
  const size_t N = v.natoms;
  int it = 0;
  if (lane == 0) it = take_unit(atomicAdd(&v.dc[DC_AGBQ], 1), nitems);
  it = __shfl_sync(FULLMASK, it, 0);
  for (; it >= 0; it = __shfl_sync(FULLMASK, it, 0)) {
    if (it >= nitems) { /* an empty cell of take_unit's table */
      if (lane == 0) it = take_unit(atomicAdd(&v.dc[DC_AGBQ], 1), nitems);
      continue;
    }
    const int4 w = items[it]; /* instance, first atom of the i block, first atom of the j run, j tiles */
    const int a1 = v.inst_begin[w.x + 1];
    const double w2 = 2.0 * v.inst_df[w.x];
    AxI I;
    AxP P;
    I.i0 = w.y + lane;
#pragma unroll
    for (int p = 0; p < AX_NP; p++) {
      float t[2][6];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int u = 2 * p + h, i = w.y + 32 * u + lane;
        const bool ok = i < a1;
        t[h][0] = ok ? -X[i] : 0.f;
        t[h][1] = ok ? -Y[i] : 0.f;
        t[h][2] = ok ? -Z[i] : 0.f;
        t[h][3] = ok ? Q[i] : 0.f;
        t[h][4] = ok ? Bv[i] : 1.f;
        t[h][5] = ok ? GbExp<float>::scale() * BI[i] : 0.f;
      }
      I.nx[p] = make_float2(t[0][0], t[1][0]);
      I.ny[p] = make_float2(t[0][1], t[1][1]);
      I.nz[p] = make_float2(t[0][2], t[1][2]);
      I.q[p] = make_float2(t[0][3], t[1][3]);
      I.b[p] = make_float2(t[0][4], t[1][4]);
      I.c[p] = make_float2(t[0][5], t[1][5]);
      P.e[p] = P.gx[p] = P.gy[p] = P.gz[p] = P.at[p] = x2(0.f);
    }
    const int iend = w.y + 64 * AX_NP;
    for (int k = 0; k < w.w; k++) {
      const int j0 = w.z + 32 * k;
      const int j = j0 + lane;
      const bool vj = j < a1;
      const float xj = vj ? X[j] : 0.f, yj = vj ? Y[j] : 0.f, zj = vj ? Z[j] : 0.f;
      const float qj = vj ? Q[j] : 0.f, bj = vj ? Bv[j] : 1.f, bij = vj ? BI[j] : 0.f;
      __syncwarp();
      sjt[wp][0][lane] = make_float4(xj, xj, yj, yj);
      sjt[wp][1][lane] = make_float4(zj, zj, qj, qj);
      sjt[wp][2][lane] = make_float4(bj, bj, bij, bij);
      __syncwarp();
      AxJ J;
      J.gx = J.gy = J.gz = J.at = x2(0.f);
      if (iend <= a1 && j0 >= iend && j0 + 32 <= a1) /* warp-uniform */
        agb_tile_x2<true>(I, P, J, sjt[wp], lane, j0, a1);
      else
        agb_tile_x2<false>(I, P, J, sjt[wp], lane, j0, a1);
      if (vj) {
        const int ja = v.slot_atom[j];
        atomicAdd(&v.g_gb[3 * ja], -w2 * (double)fold(J.gx));
        atomicAdd(&v.g_gb[3 * ja + 1], -w2 * (double)fold(J.gy));
        atomicAdd(&v.g_gb[3 * ja + 2], -w2 * (double)fold(J.gz));
        atomicAdd(&v.dera[ja], (double)fold(J.at));
      }
    }
#pragma unroll
    for (int u = 0; u < 2 * AX_NP; u++) {
      const int ia = I.i0 + 32 * u;
      if (ia >= a1) continue;
      const int p = u >> 1, h = u & 1;
      const int i = v.slot_atom[ia];
      atomicAdd(&v.eatom[N + i], C_TOKCAL * w2 * (double)lo_hi(P.e[p], h));
      atomicAdd(&v.g_gb[3 * i], w2 * (double)lo_hi(P.gx[p], h));
      atomicAdd(&v.g_gb[3 * i + 1], w2 * (double)lo_hi(P.gy[p], h));
      atomicAdd(&v.g_gb[3 * i + 2], w2 * (double)lo_hi(P.gz[p], h));
      atomicAdd(&v.dera[i], (double)lo_hi(P.at[p], h));
    }
    if (lane == 0) it = take_unit(atomicAdd(&v.dc[DC_AGBQ], 1), nitems);
  }
}

/* ------------------------------------------------------------------------ */
/* Q4 lookups without float<->int conversions (which share the special-     */
/* function unit's throughput): for 0 <= x < 2^23 the sum 2^23 + x rounded   */
/* toward minus infinity is 2^23 + floor(x), whose bit pattern is           */
/* 0x4B000000 + floor(x); the fraction x - floor(x) follows exactly.        */
/* ------------------------------------------------------------------------ */
#define X2_TWO23 8388608.f
#define X2_TWO23_BITS 0x4B000000

__device__ __forceinline__ float2 floor_frac2(float2 x, float2 &fk) {
  fk = __fadd2_rd(x, x2(X2_TWO23));
  return add2(x, fma2(fk, x2(-1.f), x2(X2_TWO23))); /* x - floor(x) */
}
__device__ __forceinline__ float2 clamp_na2(float2 x) {
  return make_float2(fminf(x.x, float(AGB_NA - 1)), fminf(x.y, float(AGB_NA - 1)));
}

/* Q4/R and its derivative in t at interval record idx (one 16-byte load,
   from shared memory when SMEM; the derivative forms of spline_d: REF the
   reference's convention, else the exact derivative of the cubic) */
template <bool REF, bool SMEM>
__device__ __forceinline__ void q4_rec(const float4 *__restrict__ tv, int idx, float t, float &q, float &fp) {
  const float4 c = SMEM ? tv[idx] : __ldg(tv + idx);
  q = fmaf(t, fmaf(t, fmaf(t, c.w, c.z), c.y), c.x);
  const float d0 = REF ? fmaf(2.f, c.w, fmaf(2.f / 3.f, c.z, c.y)) : c.y;
  const float d2 = REF ? -fmaf(3.f, c.w, 2.f * c.z) : 3.f * c.w;
  fp = fmaf(t, fmaf(t, d2, 2.f * c.z), d0);
}

/* ------------------------------------------------------------------------ */
/* Born-radius chain rule (agbnp3_cpu_simd_kernels.c:681-904), the          */
/* symmetric decomposition of k_gbders_sym in packed arithmetic: a warp     */
/* owns an i block of 4 tiles (two packed pairs per lane), the j tile sits   */
/* in shared memory with every value twice ((x,x,y,y), (z,z,rh,rh),          */
/* (rs,rs,q2,q2), (ab,ab,o1,o2); rh = 1/(h R), rs = rh sp, o1/o2 the table   */
/* offsets of the j atom's radius type in either direction).  Interior j   */
/* tiles of heavy atoms evaluate both descreening directions per pair      */
/* (HH), of hydrogens only "j descreened by i" (HX); other tiles (GEN) run  */
/* the HH arithmetic with the pairs that do not count moved out of the     */
/* tables' range.  A packed pair in a rotation step is skipped when no      */
/* lane has a pair inside the range (its terms are exactly zero).           */
/* ------------------------------------------------------------------------ */
struct GxI {
  float2 nx[AX_NP], ny[AX_NP], nz[AX_NP], rh[AX_NP], rs[AX_NP], q2[AX_NP], ab[AX_NP];
  int o1[2 * AX_NP], o2[2 * AX_NP]; /* table offsets (type * AGB_NA, type * nt * AGB_NA) - 0x4B000000 */
  int i0, a1, hh;                   /* atom of the lane in the block's first tile (u-th: i0 + 32 u), bounds */
};
struct GxP {
  float2 U[AX_NP], V[AX_NP], fx[AX_NP], fy[AX_NP], fz[AX_NP], vx[AX_NP], vy[AX_NP], vz[AX_NP];
};
struct GxJ {
  float U, V, fx, fy, fz, vx, vy, vz;
};

template <int MODE, bool REF, bool SMEM>
__device__ __forceinline__ void gbd_tile_x2(const GxI &I, GxP &P, GxJ &J, const float4 (*sj)[32], int lane, int j0,
                                            const float4 *__restrict__ tv) {
  constexpr bool TWO = MODE != GBD_HX; /* both descreening directions possible */
#pragma unroll 1
  for (int r = 0; r < 32; r++) {
    const int jj = (lane + r) & 31;
    const float4 A = sj[0][jj], B = sj[1][jj], C = sj[2][jj], D = sj[3][jj];
    const float2 jx = make_float2(A.x, A.y), jy = make_float2(A.z, A.w), jz = make_float2(B.x, B.y);
    const float2 jrh = make_float2(B.z, B.w), jrs = make_float2(C.x, C.y), jq2 = make_float2(C.z, C.w);
    const float2 jab = make_float2(D.x, D.y);
    const int o1j = __float_as_int(D.z), o2j = __float_as_int(D.w);
    float2 dx[AX_NP], dy[AX_NP], dz[AX_NP], d2[AX_NP];
#pragma unroll
    for (int p = 0; p < AX_NP; p++) {
      dx[p] = add2(jx, I.nx[p]);
      dy[p] = add2(jy, I.ny[p]);
      dz[p] = add2(jz, I.nz[p]);
      d2[p] = fma2(dz[p], dz[p], fma2(dy[p], dy[p], mul2(dx[p], dx[p])));
    }
    /* coincident atoms (d^2 = 0) contribute nothing: rare in interior
       tiles, found there by a vote */
    bool fix = MODE == GBD_GEN;
    if (MODE != GBD_GEN) {
      float2 m = d2[0];
#pragma unroll
      for (int p = 1; p < AX_NP; p++) m = mul2(m, d2[p]);
      fix = __any_sync(FULLMASK, m.x * m.y == 0.f);
    }
    const int jr = j0 + jj;
#pragma unroll
    for (int p = 0; p < AX_NP; p++) {
      float2 id = rsqrt_2(d2[p]);
      const float2 d = mul2(d2[p], id);
      float2 xh1 = mul2(d, I.rh[p]), xh2 = mul2(d, jrh);
      if (fix) {
        /* a pair that does not count (coincident; in boundary tiles also
           i >= j, beyond the instance, or hydrogen-hydrogen) and a
           direction without a heavy descreener are moved out of the tables,
           whose last record is zero: no term and no force */
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int ia = I.i0 + 32 * (2 * p + h);
          const bool hiu = MODE != GBD_GEN || ia < I.hh, hj = MODE == GBD_HH || (MODE == GBD_GEN && jr < I.hh);
          const float dd = h ? d2[p].y : d2[p].x;
          const bool ok = dd > 0.f && (MODE != GBD_GEN || (jr < I.a1 && ia < jr && (hiu || hj)));
          const float o1 = ok && hiu ? 0.f : 1e30f, o2 = ok && hj ? 0.f : 1e30f;
          if (h) {
            id.y = ok ? id.y : 0.f;
            xh1.y += o1;
            xh2.y += o2;
          } else {
            id.x = ok ? id.x : 0.f;
            xh1.x += o1;
            xh2.x += o2;
          }
        }
      }
      float mn = fminf(xh1.x, xh1.y);
      if (TWO) mn = fminf(mn, fminf(xh2.x, xh2.y));
      if (!__any_sync(FULLMASK, mn < float(AGB_NA - 1))) continue; /* exactly zero for the whole warp */
      float2 fk1;
      const float2 t1 = floor_frac2(clamp_na2(xh1), fk1);
      float2 q1, fp1;
      q4_rec<REF, SMEM>(tv, __float_as_int(fk1.x) + I.o1[2 * p] + o1j, t1.x, q1.x, fp1.x);
      q4_rec<REF, SMEM>(tv, __float_as_int(fk1.y) + I.o1[2 * p + 1] + o1j, t1.y, q1.y, fp1.y);
      P.U[p] = fma2(jq2, q1, P.U[p]);
      P.V[p] = fma2(jab, q1, P.V[p]);
      const float2 dqs1 = mul2(fp1, I.rs[p]);
      float2 ht = mul2(jq2, dqs1), ut = mul2(jab, dqs1);
      if (TWO) {
        float2 fk2;
        const float2 t2 = floor_frac2(clamp_na2(xh2), fk2);
        float2 q2, fp2;
        q4_rec<REF, SMEM>(tv, __float_as_int(fk2.x) + I.o2[2 * p] + o2j, t2.x, q2.x, fp2.x);
        q4_rec<REF, SMEM>(tv, __float_as_int(fk2.y) + I.o2[2 * p + 1] + o2j, t2.y, q2.y, fp2.y);
        J.U = fmaf(I.q2[p].x, q2.x, fmaf(I.q2[p].y, q2.y, J.U));
        J.V = fmaf(I.ab[p].x, q2.x, fmaf(I.ab[p].y, q2.y, J.V));
        const float2 dqs2 = mul2(fp2, jrs);
        ht = fma2(I.q2[p], dqs2, ht);
        ut = fma2(I.ab[p], dqs2, ut);
      }
      ht = mul2(ht, id);
      ut = mul2(ut, id);
      P.fx[p] = fma2(ht, dx[p], P.fx[p]);
      P.fy[p] = fma2(ht, dy[p], P.fy[p]);
      P.fz[p] = fma2(ht, dz[p], P.fz[p]);
      P.vx[p] = fma2(ut, dx[p], P.vx[p]);
      P.vy[p] = fma2(ut, dy[p], P.vy[p]);
      P.vz[p] = fma2(ut, dz[p], P.vz[p]);
      /* the j atom takes the opposite of both halves' terms: two fused
         multiply-adds per component */
      J.fx = fmaf(-ht.x, dx[p].x, fmaf(-ht.y, dx[p].y, J.fx));
      J.fy = fmaf(-ht.x, dy[p].x, fmaf(-ht.y, dy[p].y, J.fy));
      J.fz = fmaf(-ht.x, dz[p].x, fmaf(-ht.y, dz[p].y, J.fz));
      J.vx = fmaf(-ut.x, dx[p].x, fmaf(-ut.y, dx[p].y, J.vx));
      J.vy = fmaf(-ut.x, dy[p].x, fmaf(-ut.y, dy[p].y, J.vy));
      J.vz = fmaf(-ut.x, dz[p].x, fmaf(-ut.y, dz[p].y, J.vz));
    }
    if (TWO) {
      J.U = rot1(J.U);
      J.V = rot1(J.V);
    }
    J.fx = rot1(J.fx); J.fy = rot1(J.fy); J.fz = rot1(J.fz);
    J.vx = rot1(J.vx); J.vy = rot1(J.vy); J.vz = rot1(J.vz);
  }
}

/* one block of up to 16 warps per SM, whose warps take the items from a
   device counter (spread over the list by take_unit).  SMEM: the Q4 tables
   of the heavy descreener types (View::tabh_f) are copied into shared
   memory first (no register spills then; with the tables in global memory
   ptxas spills a few dozen bytes per thread at the 128-register cap). */
template <bool REF, bool SMEM>
__global__ void __launch_bounds__(512, 1) k_gbders_x2(View v, const int4 *__restrict__ items, int nitems) {
  constexpr int NW = 16;
  extern __shared__ float4 gbd_dyn[];
  float4(*sjt)[4][32] = reinterpret_cast<float4(*)[4][32]>(gbd_dyn); /* [NW][4][32] */
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const float *X = pa<float>(v, PA_X), *Y = pa<float>(v, PA_Y), *Z = pa<float>(v, PA_Z);
  const float *RH = pa<float>(v, PA_RH), *SP = pa<float>(v, PA_SP);
  const float *Q2 = pa<float>(v, PA_Q2AB), *AB = pa<float>(v, PA_ABRW);
  const int nt = v.ntypes;
  const float4 *tv = v.tabv_f;
  /* table offsets: (descreened type, descreener type) is record row
     d * nt + e of the full tables, d * nhv + hvslot[e] of the shared copy */
  const int ncol = SMEM ? v.nhv : nt;
  if (SMEM) {
    float4 *ts = gbd_dyn + NW * 4 * 32;
    const int nrec = nt * v.nhv * AGB_NA;
    for (int q = threadIdx.x; q < nrec; q += blockDim.x) ts[q] = __ldg(v.tabh_f + q);
    tv = ts;
    __syncthreads();
  }
  const double f4p = 1.0 / (4.0 * C_PI);
  int it = 0;
  if (lane == 0) it = take_unit(atomicAdd(&v.dc[DC_GBDQ], 1), nitems);
  it = __shfl_sync(FULLMASK, it, 0);
  for (; it >= 0; it = __shfl_sync(FULLMASK, it, 0)) {
    if (it >= nitems) { /* an empty cell of take_unit's table */
      if (lane == 0) it = take_unit(atomicAdd(&v.dc[DC_GBDQ], 1), nitems);
      continue;
    }
    const int4 w = items[it];
    const int a0 = v.inst_begin[w.x], hh = a0 + v.inst_nheavy[w.x], a1 = v.inst_begin[w.x + 1];
    const double kg = f4p * v.inst_df[w.x];
    GxI I;
    GxP P;
    I.i0 = w.y + lane;
    I.a1 = a1;
    I.hh = hh;
#pragma unroll
    for (int p = 0; p < AX_NP; p++) {
      float t[2][7];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int u = 2 * p + h, i = w.y + 32 * u + lane;
        const bool ok = i < a1;
        const float rh = ok ? RH[i] : 0.f;
        const int ti = ok ? v.slot_type[i] : 0;
        t[h][0] = ok ? -X[i] : 0.f;
        t[h][1] = ok ? -Y[i] : 0.f;
        t[h][2] = ok ? -Z[i] : 0.f;
        t[h][3] = rh;
        t[h][4] = ok ? rh * SP[i] : 0.f;
        t[h][5] = ok ? Q2[i] : 0.f;
        t[h][6] = ok ? AB[i] : 0.f;
        I.o1[u] = (SMEM ? v.hvslot[ti] : ti) * AGB_NA - X2_TWO23_BITS;
        I.o2[u] = ti * ncol * AGB_NA - X2_TWO23_BITS;
      }
      I.nx[p] = make_float2(t[0][0], t[1][0]);
      I.ny[p] = make_float2(t[0][1], t[1][1]);
      I.nz[p] = make_float2(t[0][2], t[1][2]);
      I.rh[p] = make_float2(t[0][3], t[1][3]);
      I.rs[p] = make_float2(t[0][4], t[1][4]);
      I.q2[p] = make_float2(t[0][5], t[1][5]);
      I.ab[p] = make_float2(t[0][6], t[1][6]);
      P.U[p] = P.V[p] = P.fx[p] = P.fy[p] = P.fz[p] = P.vx[p] = P.vy[p] = P.vz[p] = x2(0.f);
    }
    const bool iheavy = w.y + 64 * AX_NP <= hh; /* every i tile complete and heavy */
    for (int k = 0; k < w.w; k++) {
      const int j0 = w.z + 32 * k;
      const int j = j0 + lane;
      const bool vj = j < a1;
      const float xj = vj ? X[j] : 0.f, yj = vj ? Y[j] : 0.f, zj = vj ? Z[j] : 0.f;
      const float rhj = vj ? RH[j] : 0.f, rsj = vj ? rhj * SP[j] : 0.f;
      const float q2j = vj ? Q2[j] : 0.f, abj = vj ? AB[j] : 0.f;
      const int tj = vj ? v.slot_type[j] : 0;
      __syncwarp();
      sjt[wp][0][lane] = make_float4(xj, xj, yj, yj);
      sjt[wp][1][lane] = make_float4(zj, zj, rhj, rhj);
      sjt[wp][2][lane] = make_float4(rsj, rsj, q2j, q2j);
      sjt[wp][3][lane] = make_float4(abj, abj, __int_as_float(tj * ncol * AGB_NA),
                                     __int_as_float((SMEM ? v.hvslot[tj] : tj) * AGB_NA));
      __syncwarp();
      GxJ J;
      J.U = J.V = J.fx = J.fy = J.fz = J.vx = J.vy = J.vz = 0.f;
      /* warp-uniform tile class */
      const bool interior = iheavy && j0 >= w.y + 64 * AX_NP;
      if (interior && j0 + 32 <= hh)
        gbd_tile_x2<GBD_HH, REF, SMEM>(I, P, J, sjt[wp], lane, j0, tv);
      else if (interior && j0 >= hh && j0 + 32 <= a1)
        gbd_tile_x2<GBD_HX, REF, SMEM>(I, P, J, sjt[wp], lane, j0, tv);
      else
        gbd_tile_x2<GBD_GEN, REF, SMEM>(I, P, J, sjt[wp], lane, j0, tv);
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
    for (int u = 0; u < 2 * AX_NP; u++) {
      const int ia = I.i0 + 32 * u;
      if (ia >= a1) continue;
      const int p = u >> 1, h = u & 1;
      const int i = v.slot_atom[ia];
      atomicAdd(&v.g_gb[3 * i], kg * (double)lo_hi(P.fx[p], h));
      atomicAdd(&v.g_gb[3 * i + 1], kg * (double)lo_hi(P.fy[p], h));
      atomicAdd(&v.g_gb[3 * i + 2], kg * (double)lo_hi(P.fz[p], h));
      atomicAdd(&v.g_vw[3 * i], f4p * (double)lo_hi(P.vx[p], h));
      atomicAdd(&v.g_vw[3 * i + 1], f4p * (double)lo_hi(P.vy[p], h));
      atomicAdd(&v.g_vw[3 * i + 2], f4p * (double)lo_hi(P.vz[p], h));
      if (ia < hh) {
        atomicAdd(&v.deru[i], (double)lo_hi(P.U[p], h));
        atomicAdd(&v.derv[i], (double)lo_hi(P.V[p], h));
      }
    }
    if (lane == 0) it = take_unit(atomicAdd(&v.dc[DC_GBDQ], 1), nitems);
  }
}
