/*
 * Test-infrastructure harness around the reference AGBNP3 library.
 *
 * This translation unit textually includes the reference's agbnp3.c (from
 * the reference source tree, passed with -I by oracle/Makefile) so that the
 * file-static instance table (agbnp3.c:56) becomes reachable, and adds
 * read-only accessors for the internal state that the parity tests compare:
 * the heavy-atom near list (agbnp3.c:3978-4115), the Gaussian-overlap
 * candidate buffers of the overlap tree (agbnp3_cpu_simd_kernels.c:1064-1598),
 * the water sites (agbnp3.c:1837-2012) and per-atom intermediates.
 * It is only used by tests and by the fixture generator under tests/golden/.
 * Accessors read thread 0's workspace, so callers run the reference with
 * OMP_NUM_THREADS=1.
 */
#include "agbnp3.c"

static AGBNPdata *h_agb(int tag) {
  if (!agbnp3_tag_ok(tag)) return NULL;
  return &agbdata3_list[tag];
}

int refh_nheavy(int tag) { AGBNPdata *a = h_agb(tag); return a ? a->nheavyat : -1; }

int refh_ext2int(int tag, int *out) {
  AGBNPdata *a = h_agb(tag);
  if (!a) return -1;
  memcpy(out, a->ext2int, a->natoms * sizeof(int));
  return a->natoms;
}

/* near list of thread 0: counts[nheavy], neighbors concatenated in list order */
int refh_near_list(int tag, int *counts, int *nbrs, int cap) {
  AGBNPdata *a = h_agb(tag);
  if (!a) return -1;
  NeighList *nl = a->agbw_p[0]->near_nl;
  int n = 0;
  for (int i = 0; i < a->nheavyat; i++) {
    counts[i] = nl->nne[i];
    for (int j = 0; j < nl->nne[i]; j++) {
      if (n < cap) nbrs[n] = nl->neighl[i][j];
      n++;
    }
  }
  return n;
}

/* first n entries of the Gaussian-overlap buffers (all tree levels, in the
   reference's enumeration order): raw volume, switched volume */
int refh_gbuffers(int tag, int n, float *v3, float *v3p) {
  AGBNPdata *a = h_agb(tag);
  if (!a) return -1;
  AGBworkdata *w = a->agbw_p[0];
  if (n > w->gbuffer_size) n = w->gbuffer_size;
  memcpy(v3, w->v3, n * sizeof(float));
  memcpy(v3p, w->v3p, n * sizeof(float));
  return n;
}

int refh_nws(int tag) { AGBNPdata *a = h_agb(tag); return a ? a->agbw_p[0]->nwsat : -1; }

/* water sites: pos[3], sp, parent0, type, khb per site */
int refh_ws(int tag, float *pos, float *sp, int *parent0, int *type, int cap) {
  AGBNPdata *a = h_agb(tag);
  if (!a) return -1;
  AGBworkdata *w = a->agbw_p[0];
  int n = w->nwsat < cap ? w->nwsat : cap;
  for (int i = 0; i < n; i++) {
    WSat *s = &w->wsat[i];
    pos[3 * i] = s->pos[0];
    pos[3 * i + 1] = s->pos[1];
    pos[3 * i + 2] = s->pos[2];
    sp[i] = s->sp;
    parent0[i] = s->parent[0];
    type[i] = s->type;
  }
  return w->nwsat;
}

/* per-atom intermediates (internal order) from the master workspace:
   which: 0 volumep, 1 surf_area (raw), 2 sp, 3 spe, 4 br, 5 br1, 6 dera,
   7 deru, 8 derv, 9 derh, 10 q2ab, 11 abrw, 12 psvol, 13 gammap,
   14 derus, 15 dervs, 16 brw, 17 br1_swf_der */
int refh_atom_array(int tag, int which, float *out) {
  AGBNPdata *a = h_agb(tag);
  if (!a) return -1;
  AGBworkdata *w = a->agbw;
  float *src = NULL;
  switch (which) {
    case 0: src = w->volumep; break;
    case 1: src = w->surf_area; break;
    case 2: src = w->sp; break;
    case 3: src = w->spe; break;
    case 4: src = w->br; break;
    case 5: src = w->br1; break;
    case 6: src = w->dera; break;
    case 7: src = w->deru; break;
    case 8: src = w->derv; break;
    case 9: src = w->derh; break;
    case 10: src = w->q2ab; break;
    case 11: src = w->abrw; break;
    case 12: src = a->agbw_p[0]->psvol; break;
    case 13: src = w->gammap; break;
    case 14: src = w->derus; break;
    case 15: src = w->dervs; break;
    case 16: src = w->brw; break;
    case 17: src = w->br1_swf_der; break;
    default: return -1;
  }
  memcpy(out, src, a->natoms * sizeof(float));
  return a->natoms;
}

/* radius types and the spline table of one ordered radius-type pair */
int refh_rtypes(int tag, int *rtype) {
  AGBNPdata *a = h_agb(tag);
  if (!a) return -1;
  memcpy(rtype, a->rtype, a->natoms * sizeof(int));
  return a->nrtype;
}

int refh_table(int tag, int slot, float *y, float *y2) {
  AGBNPdata *a = h_agb(tag);
  if (!a || slot < 0 || slot >= a->nrtype * a->nrtype) return -1;
  C1Table *t = a->f4c1table2dl->table[slot];
  memcpy(y, t->y, t->n * sizeof(float));
  memcpy(y2, t->y2, t->n * sizeof(float));
  return t->n;
}
