/*
 * NeighList container used to pass the connection table to agbnp3_new().
 *
 * Drop-in for the reference's nblist.h (nblist.h:20-76): the struct layout,
 * the return codes and the three functions are the same, so callers built
 * against the reference link against this library unchanged.
 */
#ifndef LIBNBLIST_H
#define LIBNBLIST_H
#ifdef __cplusplus
extern "C" {
#endif

/* return codes (nblist.h:27-28) */
#define NBLIST_OK 0
#define NBLIST_ERR 1

typedef struct vector_ { /* a 3D vector (nblist.h:36-38) */
  double x, y, z;
} NeighVector;

/* neighbour list (nblist.h:41-70): neighbours of atom i are
   neighl[i][0 .. nne[i]-1]; neighl[i] points into neighl1 */
typedef struct neighlist_ {
  int natoms;
  int neighl_size;
  int *nne;
  int *neighl1;
  int **neighl;
  int idx_remap;
  int *int2ext;
  int *ext2int;
  int pbc;
  NeighVector *pbc_trans1;
  NeighVector **pbc_trans;
  int data;
  void **data_index1;
  void ***data_index;
} NeighList;

/* replaces nblist_reset_neighbor_list (nblist.c:30-45): sets every field to
   zero / NULL without freeing */
void nblist_reset_neighbor_list(NeighList *neigh_list);

/* replaces nblist_delete_neighbor_list (nblist.c:48-60): frees the arrays */
void nblist_delete_neighbor_list(NeighList *neigh_list);

/* replaces nblist_reallocate_neighbor_list (nblist.c:64-180): grows the
   per-atom arrays to `natoms` and the neighbour storage to `size`,
   keeping contents and rebuilding the neighl pointers; NBLIST_OK or
   NBLIST_ERR */
int nblist_reallocate_neighbor_list(NeighList *neigh_list, int natoms, int size);

#ifdef __cplusplus
}
#endif
#endif
