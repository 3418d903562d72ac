/*
 * NeighList container functions (the connection-table type of agbnp3_new).
 * Same behaviour as the reference's nblist.c:30-180: reset clears every
 * field, delete frees the arrays, reallocate grows the per-atom arrays and
 * the neighbour storage while keeping their contents and re-pointing
 * neighl[] (and the optional PBC / data arrays) into the new storage.
 */
#include <stdio.h>
#include <stdlib.h>

#include "nblist.h"

void nblist_reset_neighbor_list(NeighList *nl) {
  nl->natoms = 0;
  nl->neighl_size = 0;
  nl->nne = NULL;
  nl->neighl1 = NULL;
  nl->neighl = NULL;
  nl->idx_remap = 0;
  nl->int2ext = NULL;
  nl->ext2int = NULL;
  nl->pbc = 0;
  nl->pbc_trans1 = NULL;
  nl->pbc_trans = NULL;
  nl->data = 0;
  nl->data_index = NULL;
  nl->data_index1 = NULL;
}

void nblist_delete_neighbor_list(NeighList *nl) {
  if (!nl) return;
  free(nl->nne);
  free(nl->neighl);
  free(nl->neighl1);
  free(nl->int2ext);
  free(nl->ext2int);
  free(nl->pbc_trans);
  free(nl->pbc_trans1);
  free(nl->data_index);
  free(nl->data_index1);
}

static int grow(void **p, size_t bytes, const char *what) {
  void *q = realloc(*p, bytes ? bytes : 1);
  if (!q) {
    fprintf(stderr, "nblist_reallocate_neighbor_list(): unable to (re)allocate %s (%zu bytes).\n", what, bytes);
    return 0;
  }
  *p = q;
  return 1;
}

int nblist_reallocate_neighbor_list(NeighList *nl, int natoms, int size) {
  if (natoms > nl->natoms) {
    if (!grow((void **)&nl->nne, sizeof(int) * (size_t)natoms, "nne")) return NBLIST_ERR;
    if (!grow((void **)&nl->neighl, sizeof(int *) * (size_t)natoms, "neighl")) return NBLIST_ERR;
    if (nl->idx_remap) {
      if (!grow((void **)&nl->int2ext, sizeof(int) * (size_t)natoms, "int2ext")) return NBLIST_ERR;
      if (!grow((void **)&nl->ext2int, sizeof(int) * (size_t)natoms, "ext2int")) return NBLIST_ERR;
    }
    if (nl->pbc && !grow((void **)&nl->pbc_trans, sizeof(NeighVector *) * (size_t)natoms, "pbc_trans"))
      return NBLIST_ERR;
    if (nl->data && !grow((void **)&nl->data_index, sizeof(void **) * (size_t)natoms, "data_index"))
      return NBLIST_ERR;
  }
  if (size > nl->neighl_size) {
    if (!grow((void **)&nl->neighl1, sizeof(int) * (size_t)size, "neighl1")) return NBLIST_ERR;
    int off = 0;
    for (int i = 0; i < nl->natoms; i++) {
      nl->neighl[i] = nl->neighl1 + off;
      off += nl->nne[i];
    }
    if (nl->pbc) {
      if (!grow((void **)&nl->pbc_trans1, sizeof(NeighVector) * (size_t)size, "pbc_trans1")) return NBLIST_ERR;
      off = 0;
      for (int i = 0; i < nl->natoms; i++) {
        nl->pbc_trans[i] = nl->pbc_trans1 + off;
        off += nl->nne[i];
      }
    }
    if (nl->data) {
      if (!grow((void **)&nl->data_index1, sizeof(void *) * (size_t)size, "data_index1")) return NBLIST_ERR;
      off = 0;
      for (int i = 0; i < nl->natoms; i++) {
        nl->data_index[i] = nl->data_index1 + off;
        off += nl->nne[i];
      }
    }
    nl->neighl_size = size;
  }
  if (natoms > nl->natoms) nl->natoms = natoms;
  return NBLIST_OK;
}
