/*
 * AGBNP3 implicit-solvent model: public C API of the B200 engine.
 *
 * Drop-in for the reference's agbnp3.h (agbnp3.h:27-104): same types,
 * constants and entry points, so a caller that builds against the reference
 * header links against libagbnp3_b200.so unchanged.  The evaluation itself
 * runs on the GPU (see agbnp3_b200.h for the extensions: precision mode,
 * device-resident evaluation, batches, stage timers).
 */
#ifndef AGBNP3_H
#define AGBNP3_H

#ifdef __cplusplus
extern "C" {
#endif

#include "nblist.h"

#ifndef FALSE
#define FALSE 0
#endif
#ifndef TRUE
#define TRUE 1
#endif

/* interface floating-point type (agbnp3.h:44-50): double, or float for a
   caller built with SINGLE_PREC_INTERFACE, which links libagbnp3_b200_sp.so
   (the same engine built with that define: its entry points take float
   arrays and convert them; the evaluation is the same) */
#ifndef FLOAT_I_H
#define FLOAT_I_H
#ifdef SINGLE_PREC_INTERFACE
typedef float float_i;
#else
typedef double float_i;
#endif
#endif

/* return codes (agbnp3.h:52-57) */
#ifndef AGBNP_OK
#define AGBNP_OK (2)
#endif
#ifndef AGBNP_ERR
#define AGBNP_ERR (-1)
#endif

/* HB types (agbnp3.h:61-74) */
#define AGBNP_HB_INACTIVE (0)
#define AGBNP_HB_POLARH (1)
#define AGBNP_HB_TRIGONAL (10)
#define AGBNP_HB_TRIGONAL_S (30)
#define AGBNP_HB_TETRAHEDRAL (20)
#define AGBNP_HB_TRIGONAL1 (11)
#define AGBNP_HB_TRIGONAL2 (12)
#define AGBNP_HB_TRIGONAL_OOP (13)
#define AGBNP_HB_TETRAHEDRAL1 (21)
#define AGBNP_HB_TETRAHEDRAL2 (22)
#define AGBNP_HB_TETRAHEDRAL3 (23)

/* replaces agbnp3_initialize (agbnp3.h:77, agbnp3.c:67-93) */
int agbnp3_initialize(void);

/* replaces agbnp3_terminate (agbnp3.h:80, agbnp3.c:96-118): deletes every
   instance and releases the library's device memory */
void agbnp3_terminate(void);

/* replaces agbnp3_new (agbnp3.h:83-90, agbnp3.c:121-419).  Copies every
   input; the connection table is deep-copied and must not be NULL.  Builds
   the Q4 spline tables, the water-site topology and the device arena of the
   instance.  Returns AGBNP_OK and the instance id in *tag. */
int agbnp3_new(int *tag, int natoms, float_i *x, float_i *y, float_i *z, float_i *r, float_i *charge,
               float_i dielectric_in, float_i dielectric_out, float_i *igamma, float_i *sgamma, float_i *ialpha,
               float_i *salpha, int *hbtype, float_i *hbcorr, int nhydrogen, int *ihydrogen, NeighList *conntbl,
               int verbose);

/* replaces agbnp3_delete (agbnp3.h:93, agbnp3.c:422-487) */
int agbnp3_delete(int tag);

/* replaces agbnp3_ener (agbnp3.h:97-104, agbnp3.c:492-566): one energy and
   gradient evaluation at coordinates x, y, z (caller order).  Outputs are
   written in caller order; `init` is ignored, as in the reference. */
int agbnp3_ener(int tag, int init, float_i *x, float_i *y, float_i *z, float_i *sp, float_i *br,
                float_i *mol_volume, float_i *surf_area, float_i *egb, float_i (*dgbdr)[3], float_i *evdw,
                float_i *ecorr_vdw, float_i (*dvwdr)[3], float_i *ecav, float_i *ecorr_cav, float_i (*decav)[3],
                float_i *ehb, float_i (*dehb)[3]);

/* the spellings the reference README documents (README.md:52, 63, 146) */
int agbnp_initialize(void);
void agbnp_terminate(void);
int agbnp_delete(int tag);

#ifdef __cplusplus
}
#endif

#endif /* AGBNP3_H */
