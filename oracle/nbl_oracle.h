/*
 * nbl_oracle.h -- TEST INFRASTRUCTURE ONLY: C interface of the CPU parity
 * oracle (a restatement of the matscipy-neighbours CPU path, see
 * nbl_oracle.c).  Used by tests/, the smoke check and the CPU-baseline leg of
 * bench.py; never linked into the product library.
 */
#ifndef NBL_ORACLE_H
#define NBL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_OK 0
#define ORACLE_ZERO_VOLUME 1
#define ORACLE_RANGE 2

typedef struct {
    double len[3];      /* box width along each lattice direction */
    int32_t n[3];       /* cells per direction */
    int32_t nscan[3];   /* cells scanned each way */
    double bin[3][3];   /* bin[k] = cell row k / n[k] */
    double cutoff_sq;
} oracle_geometry_t;

typedef struct {
    int64_t npairs;
    int32_t *i;
    int32_t *j;
    double *D;       /* 3*npairs */
    double *d;
    int32_t *S;      /* 3*npairs */
    int64_t *counts; /* nat+1: exclusive prefix of per-atom counts */
} oracle_result_t;

int oracle_geometry(const double cell[9], double cutoff, oracle_geometry_t *g);

int oracle_neighbour_list(int quantities, const double origin[3],
                          const double cell[9], const double inv_cell[9],
                          const int pbc[3], int32_t nat, const double *r,
                          double cutoff, const double *per_atom_cutoff,
                          const double *per_type_cutoff_sq, int32_t ncutoffs,
                          const int32_t *types, oracle_result_t *out);

void oracle_result_free(oracle_result_t *o);

/* Row starts of an i-sorted pair list (first_neighbours.cc:15-38): seed[k]
   for k in [0, n]; -1 before the first atom with pairs, nn after the last. */
void oracle_first_neighbours(int32_t n, int64_t nn, const int32_t *i, int32_t *seed);

/* Triplets (ij, ik) of pairs sharing a first atom (triplet_list.cc:15-34).
   Returns the triplet count; writes at most `cap` of each when ij/ik are
   not NULL.  absdist == NULL: no distance filter. */
int64_t oracle_triplet_list(int32_t nfirst, const int32_t *first_i, const double *absdist,
                            double cutoff, int32_t *ij, int32_t *ik, int64_t cap);

#ifdef __cplusplus
}
#endif

#endif
