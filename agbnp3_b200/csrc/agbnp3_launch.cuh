/*
 * Launch helpers and device-wide primitives shared by the AGBNP3 kernels.
 *
 * Every stage kernel is launched through AGB_LAUNCH with a grid sized from
 * capacities fixed when the instance is created; kernels read their live
 * item counts from device memory and walk them grid-stride, so a whole
 * evaluation is a fixed sequence of launches with no host synchronisation
 * (and can be captured once into a CUDA graph).
 */
#ifndef AGBNP3_LAUNCH_CUH
#define AGBNP3_LAUNCH_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#define AGB_LAUNCH(kernel, grid, block, stream, ...) kernel<<<(grid), (block), 0, (stream)>>>(__VA_ARGS__)

/* block-cooperative loop (each index handled by one thread of the block)
   and the barrier that ends it */
#define AGB_COOP_FOR(t, n) for (int t = threadIdx.x; t < (n); t += blockDim.x)
#define AGB_SYNC() __syncthreads()
#define AGB_SHARED __shared__

#define AGB_GRID_STRIDE(i, n) \
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)(n); \
       i += (long long)gridDim.x * blockDim.x)

/* exclusive prefix sum of in[0..len) into out[0..len), len = min(*n, cap),
   read from device memory; the sum goes to *total.  `cap` is the size of
   in/out and sizes the grid; scratch holds cap/1024+2 ints. */
void agb_scan_excl(const int *in, int *out, const int *n, int *total, int cap, int *scratch, cudaStream_t s);
#define AGB_SCAN_LAUNCHES 2 /* kernels one agb_scan_excl launches */
/* the same, also writing owner[out[i] + t] = i for t < in[i] (slots of
   owner beyond owner_cap are skipped): the item each output belongs to */
void agb_scan_excl_owner(const int *in, int *out, const int *n, int *total, int cap, int *scratch, cudaStream_t s,
                         int *owner, int owner_cap);

/* out[q*nseg + k] = sum of vals[q*stride + j] for j in [seg[k], seg[k+1]),
   for q < nq; one block per (q, k), fixed reduction order */
void agb_segment_sum(const double *vals, long long stride, int nq, const int *seg, int nseg, double *out,
                     cudaStream_t s);

#endif
