/*
 * GB energy at given Born radii without any device allocation.
 *
 * Some callers cannot call cudaMalloc: host MD codes that own all device
 * memory through their own pool and forbid other allocations, or plugins
 * whose memory budget is fixed up front.  This entry point serves them: it runs
 * the GB pair stage of the engine (agbnp3_cpu_simd_kernels.c:66-151,
 * 329-460) on device arrays the caller passes, and keeps its scratch (the
 * packed float operands and the per-atom energy terms) in one file-scope
 * device array of fixed size, AGBNP3_STATIC_MAX_ATOMS atoms, which every GPU
 * that loads the library holds until the process exits.
 *
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  All calls share the array: calls that overlap
 * on the GPU (different streams, or different host threads) race on it and
 * must be serialised by the caller.  Each call rewrites every scratch entry
 * it reads, so nothing carries over between calls.
 */
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "agbnp3_launch.cuh"

#define AGBNP3_STATIC_MAX_ATOMS 32768
#define ST_BLOCK 128
#define ST_TOKCAL 332.0

struct __align__(16) st_f4 {
  float x, y, z, w;
};

/* scratch: float4 (x, y, z, q), float2 (B, 1/B), double per-atom energy */
#define ST_BYTES_F4 (16 * AGBNP3_STATIC_MAX_ATOMS)
#define ST_BYTES_F2 (8 * AGBNP3_STATIC_MAX_ATOMS)
#define ST_BYTES_E (8 * AGBNP3_STATIC_MAX_ATOMS)
static __device__ __align__(256) unsigned char g_static_scratch[ST_BYTES_F4 + ST_BYTES_F2 + ST_BYTES_E];

#define ST_MAX_DEVICES 64
/* device address of g_static_scratch per device.  Two host threads making
   their first call on the same device at once both store the same address,
   so the unsynchronised write is harmless. */
static void *st_addr[ST_MAX_DEVICES];

/* sets the library's last-error string (agbnp3_last_error) and prints it */
extern "C" void agb_host_set_error(const char *msg);

static int st_fail(const char *fmt, ...) {
  char msg[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof(msg), fmt, ap);
  va_end(ap);
  agb_host_set_error(msg);
  return -1; /* AGBNP_ERR */
}

__global__ void k_st_pack(int n, const double *x, const double *y, const double *z, const double *q,
                          const double *br, st_f4 *p4, float2 *p2) {
  AGB_GRID_STRIDE(i, n) {
    st_f4 a;
    a.x = (float)x[i];
    a.y = (float)y[i];
    a.z = (float)z[i];
    a.w = (float)q[i];
    p4[i] = a;
    p2[i] = make_float2((float)br[i], (float)(1.0 / br[i]));
  }
}

/* one thread per atom i, all partners j through shared-memory tiles;
   float pair terms, double per-tile accumulation (as k_agb_t) */
__global__ void __launch_bounds__(ST_BLOCK) k_st_pair(int n, double df, const st_f4 *__restrict__ p4,
                                                      const float2 *__restrict__ p2, double *__restrict__ eatom,
                                                      double *__restrict__ dera, double *__restrict__ grad) {
  __shared__ st_f4 s4[ST_BLOCK];
  __shared__ float2 s2[ST_BLOCK];
  int i = blockIdx.x * ST_BLOCK + threadIdx.x;
  bool act = i < n;
  st_f4 a = act ? p4[i] : st_f4{0, 0, 0, 0};
  float2 bi = act ? p2[i] : make_float2(1.f, 1.f);
  const float c = -0.25f * 1.4426950408889634f * bi.y;
  double e = 0, at = 0, gx = 0, gy = 0, gz = 0;
  for (int j0 = 0; j0 < n; j0 += ST_BLOCK) {
    int m = min(ST_BLOCK, n - j0);
    __syncthreads();
    if (threadIdx.x < m) {
      s4[threadIdx.x] = p4[j0 + threadIdx.x];
      s2[threadIdx.x] = p2[j0 + threadIdx.x];
    }
    __syncthreads();
    if (!act) continue;
    float pe = 0, pat = 0, px = 0, py = 0, pz = 0;
    for (int t = 0; t < m; t++) {
      float dx = s4[t].x - a.x, dy = s4[t].y - a.y, dz = s4[t].z - a.z;
      float d2 = dx * dx + dy * dy + dz * dz;
      if (!(d2 > 0.f)) continue;
      float bb = bi.x * s2[t].x;
      float et = exp2f(c * s2[t].y * d2);
      float f = rsqrtf(d2 + bb * et);
      float qf3 = s4[t].w * f * f * f;
      pe += s4[t].w * f;
      float mw = (1.f - 0.25f * et) * qf3;
      px += mw * dx;
      py += mw * dy;
      pz += mw * dz;
      pat += (bb + 0.25f * d2) * et * qf3;
    }
    e += pe;
    at += pat;
    gx += px;
    gy += py;
    gz += pz;
  }
  if (act) {
    double qi = a.w, w2 = 2.0 * df * qi;
    /* pair term halved (each pair is visited from both atoms) + self term */
    eatom[i] = ST_TOKCAL * (0.5 * w2 * e + df * qi * qi / (double)bi.x);
    dera[i] = qi * at;
    grad[3 * i] = ST_TOKCAL * w2 * gx;
    grad[3 * i + 1] = ST_TOKCAL * w2 * gy;
    grad[3 * i + 2] = ST_TOKCAL * w2 * gz;
  }
}

__global__ void k_st_sum(int n, const double *__restrict__ eatom, double *__restrict__ out) {
  __shared__ double sh[256];
  double s = 0;
  for (int i = threadIdx.x; i < n; i += 256) s += eatom[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

extern "C" int agbnp3_gb_energy_static(int natoms, const double *x, const double *y, const double *z,
                                       const double *charge, const double *born_radii, double dielectric_in,
                                       double dielectric_out, double *egb, double *dera, double *dgbdr,
                                       void *stream) {
  if (natoms <= 0 || natoms > AGBNP3_STATIC_MAX_ATOMS)
    return st_fail("agbnp3_gb_energy_static(): natoms = %d outside 1..%d", natoms, AGBNP3_STATIC_MAX_ATOMS);
  if (!x || !y || !z || !charge || !born_radii || !egb || !dera || !dgbdr)
    return st_fail("agbnp3_gb_energy_static(): NULL array");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= ST_MAX_DEVICES)
    return st_fail("agbnp3_gb_energy_static(): no usable current device (%s)", cudaGetErrorString(e));
  if (!st_addr[dev]) {
    /* the array's name is a host-side stand-in; its device address comes
       from the runtime, per device, with that device current.  Two host
       threads making their first call on one device at the same time both
       store the same address here, so that race is harmless. */
    void *p = NULL;
    e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p)
      return st_fail("agbnp3_gb_energy_static(): cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    st_addr[dev] = p;
  }
  unsigned char *base = (unsigned char *)st_addr[dev];
  st_f4 *p4 = (st_f4 *)base;
  float2 *p2 = (float2 *)(base + ST_BYTES_F4);
  double *eat = (double *)(base + ST_BYTES_F4 + ST_BYTES_F2);
  cudaStream_t s = (cudaStream_t)stream;
  double df = -0.5 * (1.0 / dielectric_in - 1.0 / dielectric_out);
  int nb = (natoms + ST_BLOCK - 1) / ST_BLOCK;
  k_st_pack<<<nb, ST_BLOCK, 0, s>>>(natoms, x, y, z, charge, born_radii, p4, p2);
  k_st_pair<<<nb, ST_BLOCK, 0, s>>>(natoms, df, p4, p2, eat, dera, dgbdr);
  k_st_sum<<<1, 256, 0, s>>>(natoms, eat, egb);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return st_fail("agbnp3_gb_energy_static(): launch failed: %s", cudaGetErrorString(e));
  return 2; /* AGBNP_OK */
}
