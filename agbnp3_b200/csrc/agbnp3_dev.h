/*
 * Internal C interface between the C host layer (agbnp3_host.c) and the
 * CUDA device layer (agbnp3_dev.cu).  Plain pointers and sizes only.
 *
 * A device system holds one or more independent instances ("molecules")
 * concatenated atom-wise; each instance keeps the internal atom order of
 * agbnp3_atom_reorder (agbnp3.c:739-779): heavy atoms first, hydrogens
 * last.  Inputs and outputs use each instance's external (caller) order,
 * concatenated in instance order.
 */
#ifndef AGBNP3_DEV_H
#define AGBNP3_DEV_H

#ifdef __cplusplus
extern "C" {
#endif

#define AGB_NA 512        /* spline nodes per Q4 table (agbnp3_private.h:682) */
#define AGB_MAX_ORDER 5   /* deepest overlap order (agbnp3_private.h:101) */
#define AGB_NSTAGE 12     /* timed stages, see agb_dev_stage_name */

/* water-site builders: which placement rule and which of its sites */
enum {
  WK_POLARH = 0,   /* along the donor-hydrogen bond           (agbnp3.c:2107-2150) */
  WK_TRIG1_A,      /* trigonal in-plane, opposite R-R1        (agbnp3.c:2310-2380) */
  WK_TRIG1_B,      /* trigonal in-plane, opposite R-R2                             */
  WK_TRIGS_A,      /* trigonal_s out-of-plane, +normal        (agbnp3.c:2600-2697) */
  WK_TRIGS_B,      /* trigonal_s out-of-plane, -normal                             */
  WK_OOP_A,        /* trigonal out-of-plane at 2.7 A, +normal (agbnp3.c:2815-2942) */
  WK_OOP_B,        /*                                 -normal                      */
  WK_BIS2,         /* trigonal2: opposite the bond bisector   (agbnp3.c:3027-3090) */
  WK_BIS3,         /* tetrahedral3                            (agbnp3.c:3477-3556) */
  WK_TET2_A,       /* tetrahedral2 lone pair, +out of plane   (agbnp3.c:3266-3390) */
  WK_TET2_B,       /*                        -out of plane                         */
  WK_TET1          /* tetrahedral1, anti-parallel to R-R1     (agbnp3.c:3704-3761) */
};

enum { AGB_PREC_FP64 = 0, AGB_PREC_MIXED = 1 };

/* device error word bits */
#define AGB_ERR_NL_CAP 1
#define AGB_ERR_TREE_CAP 2
#define AGB_ERR_WS_CAP 4
#define AGB_ERR_NONFINITE 8
#define AGB_ERR_CAND_CAP 16

typedef struct {
  int ninst;
  int natoms;                /* total over instances */
  const int *inst_begin;     /* [ninst+1] first atom of each instance */
  const int *inst_nheavy;    /* [ninst] */
  const double *inst_df;     /* [ninst] -0.5 (1/eps_in - 1/eps_out) */
  const float *inst_cell;    /* [ninst] cell edge of the neighbour grid (A) */
  /* per atom, internal order (global index) */
  const int *ext_of;         /* [natoms] global external position of each internal atom */
  const double *r;           /* radius + 0.5 A (agbnp3.c:210) */
  const double *charge, *igamma, *sgamma, *ialpha, *salpha;
  const int *rtype;          /* radius type (agbnp3_utils.c:808-838) */
  int ntypes;
  const double *tab;         /* ntypes^2 tables x AGB_NA nodes x {y, y2} */
  /* water sites, in the reference's creation order per instance */
  int nws;
  const int *ws_kind;        /* [nws] WK_* */
  const int *ws_parent;      /* [nws*4] global atom indices */
  const int *ws_nparent;     /* [nws] */
  const int *ws_prev;        /* [nws] atom whose spe the reference reads first for this site
                                (compat mode), -1 for a hydrogen / none (reads 0) */
  const double *ws_khb;      /* [nws] */
  const int *ws_begin;       /* [ninst+1] first site of each instance */
  int precision;             /* AGB_PREC_* */
  int compat;                /* reproduce the reference's free-volume index and spline-derivative sign */
  int device;
} agb_dev_desc;

typedef struct agb_dev agb_dev;

/* creates the device system: uploads static data and sizes the arena.
   Returns 0 or a negative error; the message is in agb_dev_last_error(). */
int agb_dev_create(const agb_dev_desc *d, agb_dev **out);
void agb_dev_destroy(agb_dev *s);
const char *agb_dev_last_error(void);

int agb_dev_set_mode(agb_dev *s, int precision, int compat);

/* host -> device copy of coordinates (external order, concatenated) */
int agb_dev_upload_coords(agb_dev *s, const double *x, const double *y, const double *z);
/* one evaluation on the device at the uploaded coordinates; outputs stay on
   the device.  Returns 0, or a negative error after checking the device
   error word (capacities are grown and the evaluation repeated on overflow). */
int agb_dev_evaluate(agb_dev *s);
/* several independent evaluations (distinct objects) issued together, each
   on its own stream, then checked one by one */
int agb_dev_evaluate_many(agb_dev *const *ss, int n);
/* pair-stage slot order: 1 = along a Hilbert curve (set from the
   coordinates of the next evaluation), 0 = identity */
int agb_dev_set_pair_order(agb_dev *s, int mode);
/* Verlet skin (A) of the near list: 0 = searched on the cell grid at every
   evaluation; > 0 = candidates within the cutoff plus skin, searched again
   when a heavy atom has moved skin/2 since the last search, filtered
   exactly at every evaluation */
int agb_dev_set_skin(agb_dev *s, double skin);
/* row sharding of one instance over ranks (one GPU each) */
int agb_dev_shard_unique_id(void *id, int nbytes);
int agb_dev_shard(agb_dev *s, int rank, int nranks, const void *id, int nbytes);
int agb_dev_shard_segment(agb_dev *s, int k);
long long agb_dev_shard_buffers(agb_dev *s, int k, double *host, int store);
/* device -> host copies of the outputs of the last evaluation (any pointer
   may be NULL).  energies: [ninst][7] egb evdw ecorr_vdw ecav ecorr_cav ehb
   mol_volume.  Gradients are AoS [natoms][3], external order. */
int agb_dev_download(agb_dev *s, double *energies, double *sp, double *br, double *surf_area, double *dgbdr,
                     double *dvwdr, double *decav, double *dehb);

/* the same with device arrays (caller order) and the caller's stream: the
   instance's work is ordered after what `stream` has queued, and `stream`
   waits for the output copies */
int agb_dev_upload_coords_dev(agb_dev *s, const double *x, const double *y, const double *z, void *stream);
int agb_dev_download_dev(agb_dev *s, double *energies, double *sp, double *br, double *surf_area, double *dgbdr,
                         double *dvwdr, double *decav, double *dehb, void *stream);

/* learned surrogate: the class of every atom from its radius (class_radii
   without the 0.5 A increment; *unmatched = atoms of no class), and the
   radial features (bf16 [natoms][160], internal order) of the coordinates of
   the last evaluation, normalised by mean / invstd when given */
int agb_dev_surrogate_classes(agb_dev *s, const double *class_radii, int nc, int *unmatched);
int agb_dev_surrogate_features(agb_dev *s, const float *mean, const float *invstd, void *out);

void *agb_dev_stream(agb_dev *s);
int agb_dev_set_timing(agb_dev *s, int enable);
int agb_dev_stage_times(agb_dev *s, double *ms, int n);
const char *agb_dev_stage_name(int i);
/* counters of the last evaluation: [0] near-list pairs, [1..4] kept
   overlaps of orders 2..5, [5] candidate overlaps, [6] water sites,
   [7] device error word, [8] kernels launched per evaluation */
int agb_dev_stats(agb_dev *s, long long *out, int n);
/* tunes the pair-stage work decomposition on the current coordinates
   (params_in NULL) or applies params_in = {nch, jb}; params_out = {nch, jb,
   invb us, agb+gbders us} */
int agb_dev_autotune(agb_dev *s, int reps, const int *params_in, int *params_out);
/* copies internal arrays of the last evaluation for parity tests */
long long agb_dev_debug_fetch(agb_dev *s, int what, void *out, long long cap);

#ifdef __cplusplus
}
#endif
#endif
