/*
 * Extensions of the AGBNP3 C API for the B200 engine.  None of these has a
 * counterpart in the reference's agbnp3.h; they expose the engine's
 * precision modes, device-resident evaluation, batches of instances,
 * per-stage timers and internals for parity testing.
 */
#ifndef AGBNP3_B200_H
#define AGBNP3_B200_H

#include "agbnp3.h"

#ifdef __cplusplus
extern "C" {
#endif

/* arithmetic of the pair, overlap and descreening stages */
#define AGBNP3_PREC_FP64 0  /* every stage in double: the plain FP64 path */
#define AGBNP3_PREC_MIXED 1 /* float pair/overlap/descreening math, double accumulation (default) */

/* compat = 1 (default) reproduces two behaviours of the reference: the
   water-site free-volume loop reads spe of the previously processed atom
   (agbnp3_cpu_simd_kernels.c:2854) and the Q4 spline derivative subtracts
   its second curvature term (agbnp3_utils.c:250-251).  compat = 0 uses each
   overlap's own atom and the exact spline derivative, so that forces are
   exactly -dE/dx. */
int agbnp3_set_mode(int tag, int precision, int compat);
int agbnp3_get_mode(int tag, int *precision, int *compat);

/* Order of the atoms inside the pair passes (no counterpart in the
   reference, whose pair loops run in its internal order).  mode 1 (the
   default; $AGBNP3_PAIR_ORDER=0 changes it): each instance's heavy atoms and
   its hydrogens are each sorted along a Hilbert curve, so that 32
   consecutive atoms form a compact cluster and a warp can skip the
   rotation steps whose pairs all lie beyond the Q4 tables' range (about a
   quarter of them in a 25,000-atom globule); the order is taken from the
   coordinates of the next evaluation and kept until this is called again
   (an MD caller may call it every few thousand steps).  mode 0: the
   internal order.  The order changes no pair and no result beyond the
   summation order of the pair sums. */
int agbnp3_pair_order(int tag, int mode);

/* Verlet skin of the heavy-atom near list, in A (no counterpart in the
   reference, which searches the list again on every call, agbnp3.c:1336).
   skin = 0 (default): the list is searched on the cell grid at every
   evaluation.  skin > 0: candidate pairs within 1.6 (ri + rj) + skin are
   kept and searched again only when a heavy atom has moved skin/2 since
   they were found; every evaluation applies the reference's float test to
   the candidates, so the near list, and every result, is the same as
   without a skin.  For MD callers whose atoms move little per step. */
int agbnp3_set_nblist_skin(int tag, double skin);

/* Row sharding of ONE instance over several GPUs, one process (rank) per
   GPU, each holding the whole instance (no counterpart in the reference,
   which runs one instance on one host's OpenMP threads).  Each rank
   evaluates every shard_n-th work item of the three pair passes
   (descreening, GB pair, chain rule) and all other stages in full; the
   pair passes' per-atom partial sums (descreening sums; A_i; U_i, V_i, the
   pair gradients and the GB pair energies) are added over the ranks by
   three NCCL all-reduces inside the evaluation, so every rank ends with
   the complete outputs.  Every rank must evaluate the same coordinates,
   collectively.
   agbnp3_shard_unique_id: an ncclUniqueId (returns its size in bytes) that
   rank 0 makes and passes to the others.  agbnp3_shard: this instance as
   rank `rank` of `nranks` with that id; id = NULL splits the work without
   a communicator, and evaluations then run only as the four segments of
   agbnp3_shard_segment (0: up to the descreening sums, 1: Born radii and GB
   pair pass, 2: the chain-rule pass, 3: the rest), the caller adding the
   partial sums of pass k over the ranks in between with
   agbnp3_shard_buffers (store 0: copy them out, concatenated; store 1: copy
   the sums back; returns the element count, host may be NULL).
   agbnp3_shard(tag, 0, 1, NULL, 0) undoes the sharding. */
int agbnp3_shard_unique_id(void *id, int nbytes);
int agbnp3_shard(int tag, int rank, int nranks, const void *id, int nbytes);
int agbnp3_shard_segment(int tag, int k);
long long agbnp3_shard_buffers(int tag, int k, double *host, int store);

/* CUDA device used by instances created afterwards (default: $AGBNP3_DEVICE,
   else $LOCAL_RANK, else 0) */
int agbnp3_set_device(int device);

/* copies coordinates (caller order) to the device without evaluating */
int agbnp3_set_coords(int tag, const double *x, const double *y, const double *z);
/* evaluates at the coordinates on the device; outputs stay on the device
   until agbnp3_get_results().  No host<->device copies. */
int agbnp3_ener_resident(int tag);
/* copies the outputs of the last evaluation (any pointer may be NULL);
   energies[7] = egb, evdw, ecorr_vdw, ecav, ecorr_cav, ehb, mol_volume */
int agbnp3_get_results(int tag, double *energies, double *sp, double *br, double *surf_area, double (*dgbdr)[3],
                       double (*dvwdr)[3], double (*decav)[3], double (*dehb)[3]);

/* one evaluation from and into DEVICE arrays on the instance's GPU (caller
   order): x, y, z [natoms]; energies [7] as in agbnp3_get_results; sp, br,
   surf_area [natoms]; gradients [natoms][3]; any output may be NULL.  The
   work is ordered after what is queued on `stream` (a cudaStream_t, NULL:
   the legacy default stream) and `stream` waits for the outputs, so a
   framework calling it on its current stream needs no host copies or
   synchronisation.  The host returns once the evaluation has finished on
   the device.  For callers that keep coordinates on the GPU (MD engines,
   PyTorch); agbnp3_ener with host arrays remains the drop-in call. */
int agbnp3_ener_device(int tag, const double *x, const double *y, const double *z, double *energies, double *sp,
                       double *br, double *surf_area, double *dgbdr, double *dvwdr, double *decav, double *dehb,
                       void *stream);

/* the CUDA stream (cudaStream_t) on which an instance's work runs */
void *agbnp3_stream(int tag);

/* per-stage device timers (CUDA events) of the next evaluations; stage
   names follow the reference's ATIMER blocks (agbnp3.c:1266-1279) */
int agbnp3_stage_timing(int tag, int enable);
int agbnp3_stage_times(int tag, double *ms, int n);
const char *agbnp3_stage_name(int stage);

/* counters of the last evaluation: [0] near-list pairs, [1..4] kept overlaps
   of orders 2..5, [5] unused, [6] water sites, [7] device error word,
   [8] kernel launches per evaluation, [9] near-list candidate searches so
   far (with a Verlet skin) */
int agbnp3_stats(int tag, long long *out, int n);

/* internal arrays of the last evaluation, for parity tests (see
   agbnp3_dev.cu, DBG_*); returns the element count or a negative value */
long long agbnp3_debug_fetch(int tag, int what, void *out, long long cap);

/* autotuner: times the pair-stage work decompositions (partner chunks of
   the descreening pass, j-tile runs of the symmetric passes) on the
   current coordinates and keeps the fastest; with $AGBNP3_TUNE_CACHE set,
   choices are read from / appended to that file, keyed by instance count
   and size bucket.  params (n <= 4): nch, jb, descreening us, pair passes us
   (-1 when taken from the cache) */
int agbnp3_autotune(int tag, int *params, int n);
int agbnp3_batch_autotune(int btag, int *params, int n);

/* message of the last error */
const char *agbnp3_last_error(void);

/* batches: several instances evaluated together in one launch sequence.
   The members keep their tags; coordinates and outputs are the members'
   arrays concatenated in member order. */
int agbnp3_batch_new(int *btag, int ntags, const int *tags);
int agbnp3_batch_delete(int btag);
int agbnp3_batch_natoms(int btag);
int agbnp3_batch_set_coords(int btag, const double *x, const double *y, const double *z);
int agbnp3_batch_ener_resident(int btag);
/* agbnp3_batch_ener_resident of nb distinct batches (1..64) at once: each
   batch's captured evaluation is launched on its own stream before any is
   waited for, so one batch's latency-bound stages (near list, overlap tree,
   water sites, tree derivatives) run beside another's pair passes.  Returns
   when all are done; results as after agbnp3_batch_ener_resident. */
int agbnp3_batches_ener_resident(int nb, const int *btags);
/* energies: [ntags][7] as in agbnp3_get_results */
int agbnp3_batch_get_results(int btag, double *energies, double *sp, double *br, double *surf_area,
                             double (*dgbdr)[3], double (*dvwdr)[3], double (*decav)[3], double (*dehb)[3]);
int agbnp3_batch_set_mode(int btag, int precision, int compat);
/* agbnp3_pair_order for a batch (every member's atoms ordered separately) */
int agbnp3_batch_pair_order(int btag, int mode);
int agbnp3_batch_set_nblist_skin(int btag, double skin);
/* agbnp3_stats for a batch (counts over all members) */
int agbnp3_batch_stats(int btag, long long *out, int n);
/* agbnp3_ener_device for a batch: arrays span all members, concatenated
   in member order; energies [7 * members] */
int agbnp3_batch_ener_device(int btag, const double *x, const double *y, const double *z, double *energies,
                             double *sp, double *br, double *surf_area, double *dgbdr, double *dvwdr, double *decav,
                             double *dehb, void *stream);
void *agbnp3_batch_stream(int btag);
int agbnp3_batch_stage_timing(int btag, int enable);
int agbnp3_batch_stage_times(int btag, double *ms, int n);

/* GB energy (self + pair, kcal/mol), its gradient at constant Born radii
   (kcal/mol/A, [natoms][3]) and the A_i terms of the Born-radius chain rule,
   for coordinates, charges and Born radii already on the device; all
   arrays are device pointers and `stream` is a cudaStream_t (NULL: the
   default stream).  It allocates no device memory: for callers that cannot
   call cudaMalloc (an MD code that owns all device memory through its own
   pool, a plugin with a fixed memory budget).  Its scratch is a static device array sized for at most 32768
   atoms, held by every GPU that loads the library until exit; larger
   systems are rejected with AGBNP_ERR.  The first call on each device
   looks the array up with that device current and should come before any
   stream capture.  Calls share the array, so calls that overlap on the GPU
   race and must be serialised by the caller.  No counterpart in the
   reference. */
int agbnp3_gb_energy_static(int natoms, const double *x, const double *y, const double *z, const double *charge,
                            const double *born_radii, double dielectric_in, double dielectric_out, double *egb,
                            double *dera, double *dgbdr, void *stream);

/* Learned surrogate inputs.  agbnp3_surrogate_classes assigns each atom
   the class whose radius (without the 0.5 A increment) is within 1e-3 A of
   its own (class_radii[nclass], nclass <= 5; *unmatched receives the number
   of atoms with no class).  agbnp3_surrogate_features writes, for the
   coordinates of the last evaluation, 160 radial features per atom (per
   neighbour class, 32 Gaussians of width 8/31 A centred at k * 8/31 A times
   a cosine cutoff at 8 A, plus the atom's own class at distance 0) as bf16
   [natoms][160] in the engine's internal order (heavy atoms first) into the
   device array `out`, each feature (x - mean) * invstd when both are given
   (device arrays [160]); the work is queued on the instance's stream
   (agbnp3_stream), without waiting.  No counterpart in the reference. */
int agbnp3_surrogate_classes(int tag, const double *class_radii, int nclass, int *unmatched);
int agbnp3_surrogate_features(int tag, const float *mean, const float *invstd, void *out);

/* C = A B^T (+ bias) on the 5th-generation tensor cores (tcgen05, FP32
   accumulation in tensor memory), the layer of the learned surrogate: device
   arrays bf16 A [M x K] (leading dimension lda), bf16 B [N x K] (ldb), fp32
   bias [N] or NULL, fp32 C [M x N] (ldc); K a multiple of 16, N <= 256,
   lda and ldb multiples of 8.  Runs on `stream` and waits for it.  Returns
   0, or -1 on bad sizes, a CUDA error or an MMA that did not complete.  No
   counterpart in the reference. */
int agbnp3_tc_gemm(const void *A, int lda, const void *B, int ldb, const float *bias, float *C, int ldc, int M, int N,
                   int K, void *stream);

/* Training and inference steps of the learned surrogate's MLP (device
   arrays, launched on `stream` without waiting; 0 or -1 on bad arguments or
   a launch error).  No counterpart in the reference.
   agbnp3_tc_gemm_async   agbnp3_tc_gemm without waiting; agbnp3_tc_error
                          synchronises `stream` and returns the tensor-core
                          error word (1: an MMA did not complete), reset = 1
                          clears it
   agbnp3_mlp_act         H = SiLU(Z) in bf16, row-major (ldh) and / or
                          transposed (Ht[col][row], ldt)
   agbnp3_mlp_act_grad    dZ = dH * SiLU'(Z) in bf16 (row-major, transposed);
                          db += column sums
   agbnp3_mlp_mse_grad    loss += scale sum (Y - T)^2; dY = 2 scale (Y - T)
                          as bf16 [rows][16] and transposed; db += sums
   agbnp3_mlp_adam        one Adam step (t >= 1) on fp32 parameters
   agbnp3_mlp_pack        fp32 W [N][K] -> bf16 W and / or bf16 W^T [K][ldt]
   agbnp3_mlp_gather      rows idx[] of bf16 samples and fp32 targets, with
                          the transposed batch */
int agbnp3_tc_gemm_async(const void *A, int lda, const void *B, int ldb, const float *bias, float *C, int ldc, int M,
                         int N, int K, void *stream);
int agbnp3_tc_error(int reset, void *stream);
int agbnp3_mlp_act(const float *Z, int rows, int n, int ldz, void *H, int ldh, void *Ht, int ldt, void *stream);
int agbnp3_mlp_act_grad(const float *dH, const float *Z, int rows, int n, void *dZ, void *dZt, int ldt, float *db,
                        void *stream);
int agbnp3_mlp_mse_grad(const float *Y, const float *T, int rows, int nout, float scale, void *dY16, void *dYt,
                        int ldt, float *db, float *loss, void *stream);
int agbnp3_mlp_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2, float eps,
                    int t, void *stream);
int agbnp3_mlp_pack(const float *W, int N, int K, void *Wb, void *Wt, int ldt, void *stream);
int agbnp3_mlp_gather(const void *X, const float *T, const long long *idx, int rows, int nin, int nout, void *Xb,
                      void *Xt, int ldt, float *Tb, void *stream);
/* Inference of the whole 160-128-128-2 SiLU network in one launch: Y [n][2]
   fp32 for bf16 rows X [n][160], bf16 weights W1 [128][160], W2 [128][128],
   W3 [2][128] (row-major) and fp32 biases, all device arrays, X and the
   weights 16-byte aligned.  The weights stay in shared memory, each layer
   is a group of tcgen05 MMAs into tensor memory and its bias and SiLU go
   straight from tensor memory into the next layer's operand.  Queued on
   `stream` (not waited for; an MMA wait that gave up surfaces through
   agbnp3_tc_error).  Returns 0, or -1 on bad arguments or a launch error.
   No counterpart in the reference. */
int agbnp3_mlp_forward(const void *X, int n, const void *W1, const float *b1, const void *W2, const float *b2,
                       const void *W3, const float *b3, float *Y, void *stream);

/* Arithmetic peaks of GPU `device` measured by the library's own
   throughput kernels (about 0.1 s): out[0] FP32 flop/s counting an FMA as
   two, out[1] FP64 flop/s, out[2] ex2 special-function op/s, out[3] the
   runtime's nominal SM clock (MHz).  The denominators of the pair stages'
   roofline.  Returns 4, or -1 on error.  No counterpart in the reference. */
int agbnp3_measure_peaks(int device, double *out, int n);

#ifdef __cplusplus
}
#endif
#endif
