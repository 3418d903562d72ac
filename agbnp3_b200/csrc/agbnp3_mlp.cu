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
