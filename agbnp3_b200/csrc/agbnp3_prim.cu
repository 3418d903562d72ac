/*
 * Device-wide exclusive scan with a device-resident length, and a
 * deterministic segmented sum.  These are the count -> scan -> emit
 * backbone of the near-list and overlap-tree stages (no atomics on any
 * index) and the final per-instance energy reductions.
 */
#include "agbnp3_launch.cuh"

#define SCAN_BLOCK 1024
#define SCAN_ITEMS 4 /* items per thread */
#define SCAN_TILE (SCAN_BLOCK * SCAN_ITEMS)

/* both phases run a fixed grid that loops over the live tiles, so a
   buffer sized for the worst case costs nothing beyond its live length */

/* phase 1: tile sums */
__global__ void k_scan_tiles(const int *__restrict__ in, const int *__restrict__ n, int cap, int *__restrict__ tile_sum) {
  __shared__ int sh[32];
  const int len = min(*n, cap);
  for (long long base = (long long)blockIdx.x * SCAN_TILE; base < len; base += (long long)gridDim.x * SCAN_TILE) {
    int s = 0;
    for (int k = 0; k < SCAN_ITEMS; k++) {
      long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
      if (i < len) s += max(in[i], 0); /* counts are never negative */
    }
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) sh[warp] = s;
    __syncthreads();
    if (warp == 0) {
      s = lane < SCAN_BLOCK / 32 ? sh[lane] : 0;
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if (lane == 0) tile_sum[base / SCAN_TILE] = s;
    }
    __syncthreads(); /* sh is reused by the next tile */
  }
}

/* sum over the block of one int per thread (sh: 32 ints of scratch,
   free on entry and on return) */
__device__ __forceinline__ int block_sum(int x, int *sh) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  if (lane == 0) sh[warp] = x;
  __syncthreads();
  int t = 0;
  if (warp == 0) {
    t = lane < SCAN_BLOCK / 32 ? sh[lane] : 0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) sh[0] = t;
  }
  __syncthreads();
  t = sh[0];
  __syncthreads();
  return t;
}

/* phase 2: scan inside each tile, offset by the sum of the tiles before it
   (each block adds those tile sums itself: a few hundred ints); the block
   of the last tile writes the total */
__global__ void k_scan_apply(const int *__restrict__ in, int *__restrict__ out, const int *__restrict__ n, int cap,
                             const int *__restrict__ tile_sum, int *__restrict__ total, int *__restrict__ owner,
                             int owner_cap) {
  __shared__ int sh[32];
  const int len = min(*n, cap);
  const long long ntiles = ((long long)len + SCAN_TILE - 1) / SCAN_TILE;
  if (len <= 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *total = 0;
    return;
  }
  for (long long base = (long long)blockIdx.x * SCAN_TILE; base < len; base += (long long)gridDim.x * SCAN_TILE) {
    const long long tile = base / SCAN_TILE;
    int p = 0;
    for (long long u = threadIdx.x; u < tile; u += SCAN_BLOCK) p += tile_sum[u];
    const int prefix = block_sum(p, sh);
    int v[SCAN_ITEMS];
    int s = 0;
    for (int k = 0; k < SCAN_ITEMS; k++) {
      long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
      v[k] = i < len ? max(in[i], 0) : 0; /* counts are never negative */
      s += v[k];
    }
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = s;
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += t;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int w = sh[lane];
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += t;
      }
      sh[lane] = w;
    }
    __syncthreads();
    int run = prefix + x - s + (warp > 0 ? sh[warp - 1] : 0);
    for (int k = 0; k < SCAN_ITEMS; k++) {
      long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
      if (i < len) {
        out[i] = run;
        /* the item each output slot belongs to (bounded by owner_cap) */
        if (owner)
          for (int t = max(0, -run); t < v[k] && run + t < owner_cap; t++) owner[run + t] = (int)i;
      }
      run += v[k];
    }
    if (tile == ntiles - 1 && threadIdx.x == SCAN_BLOCK - 1) *total = run;
    __syncthreads(); /* sh is reused by the next tile */
  }
}

void agb_scan_excl_owner(const int *in, int *out, const int *n, int *total, int cap, int *scratch, cudaStream_t s,
                         int *owner, int owner_cap) {
  int ntiles = (cap + SCAN_TILE - 1) / SCAN_TILE;
  if (ntiles < 1) ntiles = 1;
  int grid = ntiles < 148 * 2 ? ntiles : 148 * 2; /* two 1024-thread blocks per SM */
  AGB_LAUNCH(k_scan_tiles, grid, SCAN_BLOCK, s, in, n, cap, scratch);
  AGB_LAUNCH(k_scan_apply, grid, SCAN_BLOCK, s, in, out, n, cap, scratch, total, owner, owner_cap);
}

void agb_scan_excl(const int *in, int *out, const int *n, int *total, int cap, int *scratch, cudaStream_t s) {
  agb_scan_excl_owner(in, out, n, total, cap, scratch, s, nullptr, 0);
}

#define SEG_BLOCK 256
__global__ void k_segment_sum(const double *__restrict__ vals, long long stride, const int *__restrict__ seg,
                              int nseg, double *__restrict__ out) {
  __shared__ double sh[SEG_BLOCK];
  int k = blockIdx.x, q = blockIdx.y;
  const double *v = vals + (long long)q * stride;
  double s = 0.0;
  for (int j = seg[k] + threadIdx.x; j < seg[k + 1]; j += SEG_BLOCK) s += v[j];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = SEG_BLOCK / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[(long long)q * nseg + k] = sh[0];
}

void agb_segment_sum(const double *vals, long long stride, int nq, const int *seg, int nseg, double *out,
                     cudaStream_t s) {
  dim3 grid(nseg, nq);
  k_segment_sum<<<grid, SEG_BLOCK, 0, s>>>(vals, stride, seg, nseg, out);
}
