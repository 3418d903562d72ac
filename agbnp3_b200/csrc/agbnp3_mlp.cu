/*
 * Tensor-core (tcgen05) kernels of the learned surrogate: a BF16 linear
 * layer Y = X W^T with FP32 accumulation in TMEM, the building block of the
 * per-atom MLP's forward and backward passes.
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdio.h>

#include "agbnp3_tc.cuh"

#define TC_WAIT_POLLS (1 << 22) /* bound of every mbarrier wait */

/* device error word of the tensor-core kernels: 1 = an MMA wait gave up */
static __device__ int g_tc_err;

__device__ __forceinline__ void tc_flag_error() { atomicExch(&g_tc_err, 1); }

/* TMEM columns for an N-wide fp32 accumulator: a power of two >= 32 */
__host__ __device__ constexpr uint32_t tc_cols(int n) {
  return n <= 32 ? 32u : n <= 64 ? 64u : n <= 128 ? 128u : 256u;
}

#define TC_KC 32 /* K elements staged per round */

/* C[M x N] = A[M x K] B[N x K]^T (+ bias[N]), bf16 A and B row-major with
   leading dimensions lda, ldb, fp32 C with ldc.  One 128-row tile of C per
   block of 128 threads; K (a multiple of 16) is streamed through shared
   memory TC_KC at a time, accumulating in TMEM; N <= 256, B rows from N up
   to the next multiple of 16 read as zero. */
__global__ void __launch_bounds__(128) k_tc_gemm(const __nv_bfloat16 *__restrict__ A, int lda,
                                                 const __nv_bfloat16 *__restrict__ B, int ldb,
                                                 const float *__restrict__ bias, float *__restrict__ C, int ldc, int M,
                                                 int N, int K) {
  __shared__ __align__(1024) unsigned char sa[128 * TC_KC * 2];
  __shared__ __align__(1024) unsigned char sb[256 * TC_KC * 2];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * 128;
  const int NP = (N + 15) & ~15; /* MMA width */
  const uint32_t ncols = tc_cols(NP);
  if (tid == 0) tc_mbar_init(&mbar, 1);
  if (warp == 0) tc_alloc(&tslot, ncols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tslot;
  const uint32_t idesc = tc_idesc(128, NP);
  bool ok = true;
  uint32_t phase = 0;
  for (int k0 = 0; k0 < K && ok; k0 += TC_KC) {
    const int kc = min(TC_KC, K - k0); /* a multiple of 16 */
    const int kv = kc / 8;
    for (int e = tid; e < 128 * kv; e += 128) {
      int r = e / kv, k = (e % kv) * 8;
      uint4 t = make_uint4(0, 0, 0, 0);
      if (m0 + r < M) {
        const __nv_bfloat16 *src = A + (size_t)(m0 + r) * lda + k0 + k;
        __nv_bfloat16 u[8];
#pragma unroll
        for (int i = 0; i < 8; i++) u[i] = src[i];
        t = *(const uint4 *)u;
      }
      *(uint4 *)(sa + tc_off(r, k, kc)) = t;
    }
    for (int e = tid; e < NP * kv; e += 128) {
      int r = e / kv, k = (e % kv) * 8;
      uint4 t = make_uint4(0, 0, 0, 0);
      if (r < N) {
        const __nv_bfloat16 *src = B + (size_t)r * ldb + k0 + k;
        __nv_bfloat16 u[8];
#pragma unroll
        for (int i = 0; i < 8; i++) u[i] = src[i];
        t = *(const uint4 *)u;
      }
      *(uint4 *)(sb + tc_off(r, k, kc)) = t;
    }
    tc_fence_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = tc_smem_u32(sa), b0 = tc_smem_u32(sb);
      for (int kk = 0; kk < kc / 16; kk++)
        tc_mma(tmem, tc_desc(a0 + kk * 256, 128, kc * 16), tc_desc(b0 + kk * 256, 128, kc * 16), idesc,
               (k0 > 0 || kk > 0) ? 1u : 0u);
      tc_commit(&mbar);
    }
    /* the staged operands are reused by the next round: wait for the MMAs */
    bool done = tc_mbar_wait(&mbar, phase, TC_WAIT_POLLS);
    if (!done) done = tc_mbar_wait(&mbar, phase, TC_WAIT_POLLS);
    ok = __syncthreads_and(done);
    phase ^= 1u;
  }
  tc_fence_after();
  if (ok) {
    const int row = m0 + warp * 32 + lane;
    for (int c = 0; c < NP; c += 16) {
      float v[16];
      tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      if (row < M)
#pragma unroll
        for (int i = 0; i < 16; i++)
          if (c + i < N) C[(size_t)row * ldc + c + i] = v[i] + (bias ? bias[c + i] : 0.f);
    }
  } else if (tid == 0) {
    tc_flag_error();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tc_dealloc(tmem, ncols);
}

static int tc_last_error(void) {
  int e = 0;
  if (cudaMemcpyFromSymbol(&e, g_tc_err, sizeof(int)) != cudaSuccess) return -1;
  return e;
}

/* launches C = A B^T (+ bias) on `stream` without waiting; 0 or -1 on bad
   sizes or a launch error */
extern "C" int agb_tc_gemm_launch(const void *A, int lda, const void *B, int ldb, const float *bias, float *C,
                                  int ldc, int M, int N, int K, void *stream) {
  if (M <= 0 || N <= 0 || N > 256 || K <= 0 || K % 16 || lda < K || ldb < K || ldc < N || lda % 8 || ldb % 8)
    return -1;
  k_tc_gemm<<<(M + 127) / 128, 128, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)A, lda,
                                                                (const __nv_bfloat16 *)B, ldb, bias, C, ldc, M, N, K);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/* C = A B^T + bias with device arrays: bf16 A [M x K] (leading dimension
   lda), bf16 B [N x K] (ldb), fp32 bias [N] or NULL, fp32 C [M x N] (ldc);
   K a multiple of 16, N <= 256, lda and ldb multiples of 8.  Waits for the
   result.  Returns 0, or -1 on bad sizes, a CUDA error or an MMA that did
   not complete. */
extern "C" int agbnp3_tc_gemm(const void *A, int lda, const void *B, int ldb, const float *bias, float *C, int ldc,
                              int M, int N, int K, void *stream) {
  int zero = 0;
  if (cudaMemcpyToSymbolAsync(g_tc_err, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, (cudaStream_t)stream) !=
      cudaSuccess)
    return -1;
  if (agb_tc_gemm_launch(A, lda, B, ldb, bias, C, ldc, M, N, K, stream)) {
    fprintf(stderr, "agbnp3_tc_gemm(): unsupported sizes M %d N %d K %d lda %d ldb %d ldc %d\n", M, N, K, lda, ldb,
            ldc);
    return -1;
  }
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return -1;
  return tc_last_error() == 0 ? 0 : -1;
}

/* ------------------------------------------------------------------------ */
/* elementwise kernels of the MLP's training and inference                  */
/* ------------------------------------------------------------------------ */
/* z sigmoid(z), with the fast division (the result is rounded to bf16) */
__device__ __forceinline__ float silu_f(float z) { return __fdividef(z, 1.f + __expf(-z)); }
__device__ __forceinline__ float dsilu_f(float z) {
  float s = 1.f / (1.f + __expf(-z));
  return s * (1.f + z * (1.f - s));
}

#define EW_GRID(n) (int)(((n) + 255) / 256 < 148 * 32 ? ((n) + 255) / 256 : 148 * 32)
#define EW_LOOP(i, n) for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

/* H = SiLU(Z) in bf16, row-major (ldh) and / or transposed (Ht[c][row], ldt) */
__global__ void k_mlp_act(const float *Z, int rows, int n, int ldz, __nv_bfloat16 *H, int ldh, __nv_bfloat16 *Ht,
                          int ldt) {
  EW_LOOP(e, (long long)rows * n) {
    int r = (int)(e / n), c = (int)(e % n);
    __nv_bfloat16 h = __float2bfloat16(silu_f(Z[(size_t)r * ldz + c]));
    if (H) H[(size_t)r * ldh + c] = h;
    if (Ht) Ht[(size_t)c * ldt + r] = h;
  }
}

/* dZ = dH * SiLU'(Z) in bf16 (row-major and transposed); db += column sums */
__global__ void k_mlp_act_grad(const float *dH, const float *Z, int rows, int n, __nv_bfloat16 *dZ,
                               __nv_bfloat16 *dZt, int ldt, float *db) {
  EW_LOOP(e, (long long)rows * n) {
    int r = (int)(e / n), c = (int)(e % n);
    float g = dH[e] * dsilu_f(Z[e]);
    if (dZ) dZ[e] = __float2bfloat16(g);
    if (dZt) dZt[(size_t)c * ldt + r] = __float2bfloat16(g);
    if (db) atomicAdd(&db[c], g);
  }
}

/* loss += scale * sum (Y - T)^2; dY = 2 scale (Y - T) as bf16 [rows][16]
   (columns >= nout zero) and transposed [nout][ldt]; db += column sums */
__global__ void k_mlp_mse_grad(const float *Y, const float *T, int rows, int nout, float scale, __nv_bfloat16 *dY16,
                               __nv_bfloat16 *dYt, int ldt, float *db, float *loss) {
  EW_LOOP(e, (long long)rows * 16) {
    int r = (int)(e / 16), c = (int)(e % 16);
    float g = 0.f;
    if (c < nout) {
      float d = Y[(size_t)r * nout + c] - T[(size_t)r * nout + c];
      g = 2.f * scale * d;
      atomicAdd(loss, scale * d * d);
      if (db) atomicAdd(&db[c], g);
      if (dYt) dYt[(size_t)c * ldt + r] = __float2bfloat16(g);
    }
    if (dY16) dY16[e] = __float2bfloat16(g);
  }
}

/* Adam step t (1-based) on fp32 parameters */
__global__ void k_mlp_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2,
                           float eps, float c1, float c2) {
  EW_LOOP(i, n) {
    float gi = g[i];
    float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

/* fp32 W [N x K] -> bf16 W [N x K] and / or bf16 W^T [K x ldt] (columns >= N zero) */
__global__ void k_mlp_pack(const float *W, int N, int K, __nv_bfloat16 *Wb, __nv_bfloat16 *Wt, int ldt) {
  EW_LOOP(e, (long long)K * ldt) {
    int k = (int)(e / ldt), n = (int)(e % ldt);
    float w = n < N ? W[(size_t)n * K + k] : 0.f;
    if (Wt) Wt[e] = __float2bfloat16(w);
    if (Wb && n < N) Wb[(size_t)n * K + k] = __float2bfloat16(w);
  }
}

/* rows idx[] of a bf16 sample matrix X [*, nin] and fp32 targets T [*, nout]
   -> Xb [rows][nin], its transpose Xt [nin][ldt], Tb [rows][nout] */
__global__ void k_mlp_gather(const __nv_bfloat16 *X, const float *T, const long long *idx, int rows, int nin, int nout,
                             __nv_bfloat16 *Xb, __nv_bfloat16 *Xt, int ldt, float *Tb) {
  EW_LOOP(e, (long long)rows * nin) {
    int r = (int)(e / nin), c = (int)(e % nin);
    __nv_bfloat16 x = X[(size_t)idx[r] * nin + c];
    if (Xb) Xb[e] = x;
    if (Xt) Xt[(size_t)c * ldt + r] = x;
    if (c < nout) Tb[(size_t)r * nout + c] = T[(size_t)idx[r] * nout + c];
  }
}

#define EW_RET return cudaGetLastError() == cudaSuccess ? 0 : -1

extern "C" int agbnp3_mlp_act(const float *Z, int rows, int n, int ldz, void *H, int ldh, void *Ht, int ldt,
                              void *stream) {
  k_mlp_act<<<EW_GRID((long long)rows * n), 256, 0, (cudaStream_t)stream>>>(Z, rows, n, ldz, (__nv_bfloat16 *)H, ldh,
                                                                          (__nv_bfloat16 *)Ht, ldt);
  EW_RET;
}

extern "C" int agbnp3_mlp_act_grad(const float *dH, const float *Z, int rows, int n, void *dZ, void *dZt, int ldt,
                                   float *db, void *stream) {
  k_mlp_act_grad<<<EW_GRID((long long)rows * n), 256, 0, (cudaStream_t)stream>>>(
      dH, Z, rows, n, (__nv_bfloat16 *)dZ, (__nv_bfloat16 *)dZt, ldt, db);
  EW_RET;
}

extern "C" int agbnp3_mlp_mse_grad(const float *Y, const float *T, int rows, int nout, float scale, void *dY16,
                                   void *dYt, int ldt, float *db, float *loss, void *stream) {
  if (nout > 16) return -1;
  k_mlp_mse_grad<<<EW_GRID((long long)rows * 16), 256, 0, (cudaStream_t)stream>>>(
      Y, T, rows, nout, scale, (__nv_bfloat16 *)dY16, (__nv_bfloat16 *)dYt, ldt, db, loss);
  EW_RET;
}

extern "C" int agbnp3_mlp_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1,
                               float b2, float eps, int t, void *stream) {
  float c1 = 1.f / (1.f - powf(b1, (float)t)), c2 = 1.f / (1.f - powf(b2, (float)t));
  k_mlp_adam<<<EW_GRID(n), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
  EW_RET;
}

extern "C" int agbnp3_mlp_pack(const float *W, int N, int K, void *Wb, void *Wt, int ldt, void *stream) {
  if (ldt < N) return -1;
  k_mlp_pack<<<EW_GRID((long long)K * ldt), 256, 0, (cudaStream_t)stream>>>(W, N, K, (__nv_bfloat16 *)Wb,
                                                                           (__nv_bfloat16 *)Wt, ldt);
  EW_RET;
}

extern "C" int agbnp3_mlp_gather(const void *X, const float *T, const long long *idx, int rows, int nin, int nout,
                                 void *Xb, void *Xt, int ldt, float *Tb, void *stream) {
  if (nout > nin) return -1;
  k_mlp_gather<<<EW_GRID((long long)rows * nin), 256, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16 *)X, T, idx, rows, nin, nout, (__nv_bfloat16 *)Xb, (__nv_bfloat16 *)Xt, ldt, Tb);
  EW_RET;
}

/* ------------------------------------------------------------------------ */
/* fused inference: all three layers of the 160-128-128-2 SiLU network in   */
/* one kernel.  A block of 256 threads keeps the bf16 weights in shared     */
/* memory (canonical K-major layout) and walks 128-row tiles of the input: */
/* X tile -> smem; layer 1 (10 MMAs of K = 16) into TMEM columns 0..127;    */
/* bias + SiLU per row (two threads a row, tcgen05.ld), bf16 into H in      */
/* smem; layer 2 (8 MMAs) into columns 128..255; bias + SiLU into H again;  */
/* layer 3 (N padded to 16, 8 MMAs) into columns 0..15; bias, two outputs   */
/* per row to global memory.  Every MMA group completes through an          */
/* mbarrier with a bounded wait (error word, no result, TMEM freed).        */
/* ------------------------------------------------------------------------ */
#define MF_IN 160
#define MF_H 128
#define MF_OUT 2
#define MF_N3 16 /* layer-3 MMA width (rows >= MF_OUT of W3 are zero) */
#define MF_SMEM_W1 (MF_H * MF_IN * 2)
#define MF_SMEM_W2 (MF_H * MF_H * 2)
#define MF_SMEM_W3 (MF_N3 * MF_H * 2)
#define MF_SMEM_X (128 * MF_IN * 2)
#define MF_SMEM_H (128 * MF_H * 2)
#define MF_SMEM (MF_SMEM_W1 + MF_SMEM_W2 + MF_SMEM_W3 + MF_SMEM_X + MF_SMEM_H + 1024)

/* rows [0, rows) of a row-major bf16 matrix (leading dimension ld, `valid`
   rows present, the rest zero) into the canonical K-major layout of an
   rows x K tile; 16-byte chunks, one per thread per step */
__device__ __forceinline__ void mf_stage(unsigned char *dst, const __nv_bfloat16 *__restrict__ src, int ld, int rows,
                                         int valid, int K) {
  const int kv = K / 8;
  for (int e = threadIdx.x; e < rows * kv; e += blockDim.x) {
    const int r = e / kv, k = (e % kv) * 8;
    uint4 t = make_uint4(0, 0, 0, 0);
    if (r < valid) t = *(const uint4 *)(src + (size_t)r * ld + k);
    *(uint4 *)(dst + tc_off(r, k, K)) = t;
  }
}

/* half a row of fp32 accumulators (TMEM columns c0..c0+63 of this thread's
   lane, taddr = the lane's column 0) -> bias + SiLU -> bf16 into row r of
   the H tile */
__device__ __forceinline__ void mf_act_row(uint32_t taddr, const float *__restrict__ bias, unsigned char *h, int r,
                                           int c0) {
#pragma unroll 1
  for (int c = c0; c < c0 + MF_H / 2; c += 16) {
    float v[16];
    tc_ld16(taddr + (uint32_t)c, v);
#pragma unroll
    for (int half = 0; half < 2; half++) {
      __align__(16) __nv_bfloat16 u[8];
#pragma unroll
      for (int i = 0; i < 8; i++) u[i] = __float2bfloat16(silu_f(v[8 * half + i] + bias[c + 8 * half + i]));
      *(uint4 *)(h + tc_off(r, c + 8 * half, MF_H)) = *(const uint4 *)u;
    }
  }
}

/* waits for the mbarrier phase (bounded) and agrees on the outcome */
__device__ __forceinline__ bool mf_wait(uint64_t *mbar, uint32_t &phase) {
  bool done = tc_mbar_wait(mbar, phase, TC_WAIT_POLLS);
  if (!done) done = tc_mbar_wait(mbar, phase, TC_WAIT_POLLS);
  phase ^= 1u;
  return __syncthreads_and(done);
}

#define MF_THREADS 256 /* warps w and w + 4 read TMEM lanes 32 (w % 4) .. + 31, each half of the columns */
__global__ void __launch_bounds__(MF_THREADS, 1) k_mlp_fwd(const __nv_bfloat16 *__restrict__ X, int n,
                                                    const __nv_bfloat16 *__restrict__ W1, const float *__restrict__ b1,
                                                    const __nv_bfloat16 *__restrict__ W2, const float *__restrict__ b2,
                                                    const __nv_bfloat16 *__restrict__ W3, const float *__restrict__ b3,
                                                    float *__restrict__ Y) {
  extern __shared__ unsigned char mf_raw[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  unsigned char *base = (unsigned char *)(((uintptr_t)mf_raw + 1023) & ~(uintptr_t)1023);
  unsigned char *sw1 = base, *sw2 = sw1 + MF_SMEM_W1, *sw3 = sw2 + MF_SMEM_W2, *sx = sw3 + MF_SMEM_W3,
                *sh = sx + MF_SMEM_X;
  const int tid = threadIdx.x, warp = tid >> 5, quad = warp & 3, r = 32 * quad + (tid & 31);
  const int c0 = (warp >> 2) * (MF_H / 2); /* this thread's half of the columns */
  mf_stage(sw1, W1, MF_IN, MF_H, MF_H, MF_IN);
  mf_stage(sw2, W2, MF_H, MF_H, MF_H, MF_H);
  mf_stage(sw3, W3, MF_H, MF_N3, MF_OUT, MF_H);
  if (tid == 0) tc_mbar_init(&mbar, 1);
  if (warp == 0) tc_alloc(&tslot, 256);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tslot, lane_off = (uint32_t)(quad * 32) << 16;
  const uint32_t id1 = tc_idesc(128, MF_H), id3 = tc_idesc(128, MF_N3);
  const uint32_t aw1 = tc_smem_u32(sw1), aw2 = tc_smem_u32(sw2), aw3 = tc_smem_u32(sw3), ax = tc_smem_u32(sx),
                 ah = tc_smem_u32(sh);
  uint32_t phase = 0;
  bool ok = true;
  for (int m0 = blockIdx.x * 128; m0 < n && ok; m0 += gridDim.x * 128) {
    const int row = m0 + r; /* this thread's row: TMEM lane r */
    mf_stage(sx, X + (size_t)m0 * MF_IN, MF_IN, 128, min(128, n - m0), MF_IN);
    tc_fence_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      for (int kk = 0; kk < MF_IN / 16; kk++)
        tc_mma(tmem, tc_desc(ax + kk * 256, 128, MF_IN * 16), tc_desc(aw1 + kk * 256, 128, MF_IN * 16), id1,
               kk > 0 ? 1u : 0u);
      tc_commit(&mbar);
    }
    if (!(ok = mf_wait(&mbar, phase))) break;
    tc_fence_after();
    mf_act_row(tmem + lane_off, b1, sh, r, c0);
    tc_fence_before();
    tc_fence_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      for (int kk = 0; kk < MF_H / 16; kk++)
        tc_mma(tmem + 128, tc_desc(ah + kk * 256, 128, MF_H * 16), tc_desc(aw2 + kk * 256, 128, MF_H * 16), id1,
               kk > 0 ? 1u : 0u);
      tc_commit(&mbar);
    }
    if (!(ok = mf_wait(&mbar, phase))) break;
    tc_fence_after();
    mf_act_row(tmem + lane_off + 128, b2, sh, r, c0);
    tc_fence_before();
    tc_fence_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      for (int kk = 0; kk < MF_H / 16; kk++)
        tc_mma(tmem, tc_desc(ah + kk * 256, 128, MF_H * 16), tc_desc(aw3 + kk * 256, 128, MF_H * 16), id3,
               kk > 0 ? 1u : 0u);
      tc_commit(&mbar);
    }
    if (!(ok = mf_wait(&mbar, phase))) break;
    tc_fence_after();
    if (warp < 4) {
      float v[16];
      tc_ld16(tmem + lane_off, v);
      if (row < n) {
        Y[(size_t)row * MF_OUT] = v[0] + b3[0];
        Y[(size_t)row * MF_OUT + 1] = v[1] + b3[1];
      }
    }
    tc_fence_before();
    __syncthreads(); /* TMEM and the X tile are reused by the next tile */
  }
  if (!ok && tid == 0) tc_flag_error();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tc_dealloc(tmem, 256);
}

/* Y [n x 2] fp32 = the 160-128-128-2 SiLU network applied to the bf16 rows
   of X [n x 160] (row-major), with bf16 weights W1 [128 x 160], W2
   [128 x 128], W3 [2 x 128] (row-major, as nn.Linear stores them) and fp32
   biases, in one launch on `stream` (not waited for; a wait that gave up
   surfaces through agbnp3_tc_error).  X and the weights must be 16-byte
   aligned.  Returns 0, or -1 on bad arguments or a launch error. */
extern "C" int agbnp3_mlp_forward(const void *X, int n, const void *W1, const float *b1, const void *W2,
                                  const float *b2, const void *W3, const float *b3, float *Y, void *stream) {
  /* the shared-memory limit is raised once per device (an attribute of the
     function on the current device); setting it twice is harmless */
  static int attr_set[64];
  if (n <= 0 || !X || !W1 || !b1 || !W2 || !b2 || !W3 || !b3 || !Y) return -1;
  if (((uintptr_t)X | (uintptr_t)W1 | (uintptr_t)W2 | (uintptr_t)W3) & 15) return -1;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
  if (!attr_set[dev]) {
    if (cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, MF_SMEM) != cudaSuccess)
      return -1;
    attr_set[dev] = 1;
  }
  int tiles = (n + 127) / 128, grid = tiles < 148 ? tiles : 148;
  k_mlp_fwd<<<grid, MF_THREADS, MF_SMEM, (cudaStream_t)stream>>>(
      (const __nv_bfloat16 *)X, n, (const __nv_bfloat16 *)W1, b1, (const __nv_bfloat16 *)W2, b2,
      (const __nv_bfloat16 *)W3, b3, Y);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/* the GEMM without waiting, for the training loop (errors surface through
   agbnp3_tc_error) */
extern "C" int agbnp3_tc_gemm_async(const void *A, int lda, const void *B, int ldb, const float *bias, float *C,
                                    int ldc, int M, int N, int K, void *stream) {
  return agb_tc_gemm_launch(A, lda, B, ldb, bias, C, ldc, M, N, K, stream);
}

/* the tensor-core error word (1: an MMA wait gave up since the last reset),
   read after synchronising `stream`; reset = 1 clears it */
extern "C" int agbnp3_tc_error(int reset, void *stream) {
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return -1;
  int e = tc_last_error();
  if (reset) {
    int zero = 0;
    cudaMemcpyToSymbol(g_tc_err, &zero, sizeof(int));
  }
  return e;
}
