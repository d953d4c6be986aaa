/*
 * nbl_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity oracle).
 *
 * A plain-C restatement of the matscipy-neighbours CPU neighbour-list path,
 * used by the test-suite, the smoke check and the CPU-baseline leg of the
 * benchmark as the checker.  Nothing in the shipped library links or calls it.
 *
 * Arithmetic contract (what makes this an oracle and not "a" neighbour list):
 * every floating-point step is done in the same order and with the same
 * roundings as the reference C++ core compiled for x86-64 without FMA
 * (the recipe in oracle/Makefile builds this file with -ffp-contract=off).
 * Pinned against the reference's own core (oracle/_ref, built from the
 * reference sources by oracle/Makefile) and against the reference's
 * known-answer tests; see tests/test_oracle.py.
 *
 * Reference files followed (paths inside the reference project):
 *   src/libneighbours/tools.hh:30-67          mat_mul_vec, bin_wrap, bin_trunc,
 *                                             position_to_cell_index
 *   src/libneighbours/tools.cc:17-25          cross_product, norm
 *   src/libneighbours/cell_list.cc:153-182    cell_grid_geometry
 *   src/libneighbours/cell_list.cc:23-102     folded coords + stable binning
 *   src/libneighbours/neighbour_list.cc:99-204   driver (raw cells, gather,
 *                                             context, two passes)
 *   src/libneighbours/neighbour_visit.hh:51-120  visit_neighbours
 *
 * Binning: the reference sorts atoms into cells with a stable counting sort
 * (dense grid) or a stable serial scatter into a hash table (sparse grid);
 * both leave the atoms of one cell in ascending original-index order, and the
 * traversal visits neighbour cells by offset, so the order in which cells sit
 * in memory never reaches the output.  This restatement therefore sorts atoms
 * stably by their 64-bit linear cell key and looks cells up by binary search,
 * which is valid for both reference backends.
 */

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "nbl_oracle.h"

/* Quantity bits as in src/libneighbours/types.hh:38-44. */
#define Q_I 1
#define Q_J 2
#define Q_D 4
#define Q_d 8
#define Q_S 16

/* x86-64 cvttsd2si semantics for double -> int32 (used by the reference's
   static_cast<int>(floor(..)) in cell_list.cc:167-169): out of range or NaN
   gives INT32_MIN. */
static int32_t x86_trunc_i32(double v) {
    if (!(v > -2147483649.0 && v < 2147483648.0)) return INT32_MIN;
    return (int32_t)v;
}

/* tools.hh:43-46 (periodic wrap), computed by modulo instead of a loop. */
static int32_t wrap_cell(int32_t i, int32_t n) {
    int32_t r = i % n;
    return r < 0 ? r + n : r;
}

/* tools.hh:49-56 (non-periodic clamp). */
static int32_t trunc_cell(int32_t i, int32_t n) {
    if (i < 0) return 0;
    if (i >= n) return n - 1;
    return i;
}

static void cross3(const double *a, const double *b, double *c) {
    /* tools.cc:17-21 */
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

static double norm3(const double *a) {
    /* tools.cc:23-25 */
    return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
}

int oracle_geometry(const double cell[9], double cutoff, oracle_geometry_t *g) {
    /* cell_list.cc:153-182 */
    const double *c1 = &cell[0], *c2 = &cell[3], *c3 = &cell[6];
    double nrm1[3], nrm2[3], nrm3[3];
    cross3(c2, c3, nrm1);
    cross3(c3, c1, nrm2);
    cross3(c1, c2, nrm3);
    double vol = fabs(c3[0] * nrm3[0] + c3[1] * nrm3[1] + c3[2] * nrm3[2]);
    if (vol < 1e-12) return ORACLE_ZERO_VOLUME;
    g->len[0] = vol / norm3(nrm1);
    g->len[1] = vol / norm3(nrm2);
    g->len[2] = vol / norm3(nrm3);
    for (int k = 0; k < 3; k++) {
        int32_t n = x86_trunc_i32(floor(g->len[k] / cutoff));
        g->n[k] = n > 1 ? n : 1;
    }
    for (int k = 0; k < 3; k++) {
        g->bin[0][k] = c1[k] / g->n[0];
        g->bin[1][k] = c2[k] / g->n[1];
        g->bin[2][k] = c3[k] / g->n[2];
    }
    /* neighbour_list.cc:174-176: cells to scan each way. */
    for (int k = 0; k < 3; k++) {
        double s = cutoff * g->n[k] / g->len[k];
        g->nscan[k] = (int32_t)ceil(s);
    }
    g->cutoff_sq = cutoff * cutoff;
    return ORACLE_OK;
}

typedef struct {
    int64_t key;
    int32_t atom;
} keyed_atom;

static int cmp_keyed(const void *pa, const void *pb) {
    const keyed_atom *a = (const keyed_atom *)pa, *b = (const keyed_atom *)pb;
    if (a->key != b->key) return a->key < b->key ? -1 : 1;
    return a->atom < b->atom ? -1 : (a->atom > b->atom ? 1 : 0);
}

/* Cell lookup: [begin,end) of the atoms of the cell with linear key `key`. */
static void cell_slice(const int64_t *ukey, const int32_t *ufirst, int64_t nu,
                       int64_t key, int32_t *b, int32_t *e) {
    int64_t lo = 0, hi = nu;
    while (lo < hi) {
        int64_t mid = (lo + hi) / 2;
        if (ukey[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    if (lo < nu && ukey[lo] == key) {
        *b = ufirst[lo];
        *e = ufirst[lo + 1];
    } else {
        *b = 0;
        *e = 0;
    }
}

typedef struct {
    int32_t n[3];
    int32_t nscan[3];
    int pbc[3];
    double bin[3][3];
    double cutoff_sq;
    const double *per_type_sq;
    int32_t ncutoffs;
    const int32_t *raw;     /* 3*nat, sorted */
    const int32_t *rel;     /* 3*nat, sorted */
    const double *pos;      /* 3*nat, sorted, bin-relative */
    const double *per_atom; /* nat, sorted, or NULL */
    const int32_t *types;   /* nat, sorted, or NULL */
    const int64_t *ukey;
    const int32_t *ufirst;
    int64_t nu;
} visit_ctx;

/* neighbour_visit.hh:51-120.  `sink` is called per neighbour (count or fill). */
typedef void (*emit_fn)(void *state, int32_t sj, const double dr[3], double r2,
                        const int32_t shift[3]);

static void visit(const visit_ctx *c, int32_t si, emit_fn emit, void *state) {
    const int32_t n1 = c->n[0], n2 = c->n[1], n3 = c->n[2];
    const int32_t *raw_i = &c->raw[3 * si];
    const double *pi = &c->pos[3 * si];
    const int32_t ci1 = c->pbc[0] ? wrap_cell(raw_i[0], n1) : trunc_cell(raw_i[0], n1);
    const int32_t ci2 = c->pbc[1] ? wrap_cell(raw_i[1], n2) : trunc_cell(raw_i[1], n2);
    const int32_t ci3 = c->pbc[2] ? wrap_cell(raw_i[2], n3) : trunc_cell(raw_i[2], n3);

    for (int32_t z = -c->nscan[2]; z <= c->nscan[2]; z++) {
        int32_t cj3 = ci3 + z;
        if (c->pbc[2]) cj3 = wrap_cell(cj3, n3);
        if (cj3 < 0 || cj3 >= n3) continue;
        double o3[3] = {z * c->bin[2][0], z * c->bin[2][1], z * c->bin[2][2]};
        for (int32_t y = -c->nscan[1]; y <= c->nscan[1]; y++) {
            int32_t cj2 = ci2 + y;
            if (c->pbc[1]) cj2 = wrap_cell(cj2, n2);
            if (cj2 < 0 || cj2 >= n2) continue;
            double o2[3] = {o3[0] + y * c->bin[1][0], o3[1] + y * c->bin[1][1],
                            o3[2] + y * c->bin[1][2]};
            for (int32_t x = -c->nscan[0]; x <= c->nscan[0]; x++) {
                int32_t cj1 = ci1 + x;
                if (c->pbc[0]) cj1 = wrap_cell(cj1, n1);
                if (cj1 < 0 || cj1 >= n1) continue;
                double o[3] = {o2[0] + x * c->bin[0][0], o2[1] + x * c->bin[0][1],
                               o2[2] + x * c->bin[0][2]};
                int64_t key = (int64_t)cj1 +
                              (int64_t)n1 * ((int64_t)cj2 + (int64_t)n2 * cj3);
                int32_t b, e;
                cell_slice(c->ukey, c->ufirst, c->nu, key, &b, &e);
                for (int32_t sj = b; sj < e; sj++) {
                    if (sj == si && x == 0 && y == 0 && z == 0) continue;
                    const double *pj = &c->pos[3 * sj];
                    double dr[3] = {pj[0] - pi[0] + o[0], pj[1] - pi[1] + o[1],
                                    pj[2] - pi[2] + o[2]};
                    double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
                    if (r2 >= c->cutoff_sq) continue;
                    int inside = 1;
                    if (c->per_atom) {
                        double cc = c->per_atom[si] + c->per_atom[sj];
                        inside = r2 < cc * cc;
                    } else if (c->per_type_sq && c->types) {
                        int32_t ti = c->types[si], tj = c->types[sj];
                        if (ti >= 0 && ti < c->ncutoffs && tj >= 0 && tj < c->ncutoffs)
                            inside = r2 < c->per_type_sq[ti * c->ncutoffs + tj];
                    }
                    if (!inside) continue;
                    const int32_t *rj = &c->rel[3 * sj];
                    int32_t sh[3] = {(raw_i[0] - rj[0] + x) / n1,
                                     (raw_i[1] - rj[1] + y) / n2,
                                     (raw_i[2] - rj[2] + z) / n3};
                    emit(state, sj, dr, r2, sh);
                }
            }
        }
    }
}

static void emit_count(void *state, int32_t sj, const double dr[3], double r2,
                       const int32_t sh[3]) {
    (void)sj; (void)dr; (void)r2; (void)sh;
    (*(int64_t *)state)++;
}

typedef struct {
    int32_t i;
    int64_t w;
    const int32_t *sorted_atom;
    oracle_result_t *out;
} fill_state;

static void emit_fill(void *state, int32_t sj, const double dr[3], double r2,
                      const int32_t sh[3]) {
    /* neighbour_list.cc:69-94 */
    fill_state *f = (fill_state *)state;
    oracle_result_t *o = f->out;
    const int64_t w = f->w;
    if (o->i) o->i[w] = f->i;
    if (o->j) o->j[w] = f->sorted_atom[sj];
    if (o->D) {
        o->D[3 * w + 0] = dr[0];
        o->D[3 * w + 1] = dr[1];
        o->D[3 * w + 2] = dr[2];
    }
    if (o->d) o->d[w] = sqrt(r2);
    if (o->S) {
        o->S[3 * w + 0] = sh[0];
        o->S[3 * w + 1] = sh[1];
        o->S[3 * w + 2] = sh[2];
    }
    f->w = w + 1;
}

void oracle_result_free(oracle_result_t *o) {
    free(o->i);
    free(o->j);
    free(o->D);
    free(o->d);
    free(o->S);
    free(o->counts);
    memset(o, 0, sizeof(*o));
}

int oracle_neighbour_list(int quantities, const double origin[3],
                          const double cell[9], const double inv_cell[9],
                          const int pbc[3], int32_t nat, const double *r,
                          double cutoff, const double *per_atom_cutoff,
                          const double *per_type_cutoff_sq, int32_t ncutoffs,
                          const int32_t *types, oracle_result_t *out) {
    memset(out, 0, sizeof(*out));
    oracle_geometry_t g;
    if (oracle_geometry(cell, cutoff, &g) != ORACLE_OK) return ORACLE_ZERO_VOLUME;
    out->counts = (int64_t *)calloc((size_t)nat + 1, sizeof(int64_t));
    if (nat <= 0) return ORACLE_OK;

    int32_t *raw = (int32_t *)malloc(sizeof(int32_t) * 3 * (size_t)nat);
    keyed_atom *ka = (keyed_atom *)malloc(sizeof(keyed_atom) * (size_t)nat);

    /* neighbour_list.cc:126-133 with tools.hh:55-67 */
    for (int32_t a = 0; a < nat; a++) {
        double d[3], s[3];
        for (int k = 0; k < 3; k++) d[k] = r[3 * a + k] - origin[k];
        for (int k = 0; k < 3; k++) {
            s[k] = 0.0;
            for (int m = 0; m < 3; m++) s[k] += inv_cell[3 * k + m] * d[m];
        }
        for (int k = 0; k < 3; k++) {
            double f = floor(s[k] * g.n[k]);
            /* Outside +-2^29 cells (or NaN) the reference's int conversion and
               shift arithmetic are undefined; the product rejects such input
               with a range error and so does the oracle. */
            if (!(f > -536870912.0 && f < 536870912.0)) {
                free(raw);
                free(ka);
                return ORACLE_RANGE;
            }
            raw[3 * a + k] = (int32_t)f;
        }
    }
    /* cell_list.cc:23-41 (fold) and the linear key of cell_list.cc:55-57 */
    for (int32_t a = 0; a < nat; a++) {
        int32_t c[3];
        for (int k = 0; k < 3; k++)
            c[k] = pbc[k] ? wrap_cell(raw[3 * a + k], g.n[k])
                          : trunc_cell(raw[3 * a + k], g.n[k]);
        ka[a].key = (int64_t)c[0] +
                    (int64_t)g.n[0] * ((int64_t)c[1] + (int64_t)g.n[1] * c[2]);
        ka[a].atom = a;
    }
    qsort(ka, (size_t)nat, sizeof(keyed_atom), cmp_keyed);

    int64_t nu = 0;
    int64_t *ukey = (int64_t *)malloc(sizeof(int64_t) * (size_t)nat);
    int32_t *ufirst = (int32_t *)malloc(sizeof(int32_t) * ((size_t)nat + 1));
    for (int32_t s = 0; s < nat; s++) {
        if (s == 0 || ka[s].key != ka[s - 1].key) {
            ukey[nu] = ka[s].key;
            ufirst[nu] = s;
            nu++;
        }
    }
    ufirst[nu] = nat;

    /* neighbour_list.cc:139-167: per-atom data in cell-sorted order. */
    int32_t *sorted_atom = (int32_t *)malloc(sizeof(int32_t) * (size_t)nat);
    int32_t *raw_s = (int32_t *)malloc(sizeof(int32_t) * 3 * (size_t)nat);
    int32_t *rel_s = (int32_t *)malloc(sizeof(int32_t) * 3 * (size_t)nat);
    double *pos_s = (double *)malloc(sizeof(double) * 3 * (size_t)nat);
    double *pa_s = per_atom_cutoff ? (double *)malloc(sizeof(double) * (size_t)nat) : NULL;
    int32_t *ty_s = types ? (int32_t *)malloc(sizeof(int32_t) * (size_t)nat) : NULL;
    for (int32_t s = 0; s < nat; s++) {
        const int32_t a = ka[s].atom;
        sorted_atom[s] = a;
        int32_t rc[3];
        for (int k = 0; k < 3; k++) {
            raw_s[3 * s + k] = raw[3 * a + k];
            rc[k] = pbc[k] ? raw[3 * a + k] : trunc_cell(raw[3 * a + k], g.n[k]);
            rel_s[3 * s + k] = rc[k];
        }
        for (int k = 0; k < 3; k++)
            pos_s[3 * s + k] = r[3 * a + k] - rc[0] * g.bin[0][k] -
                               rc[1] * g.bin[1][k] - rc[2] * g.bin[2][k];
        if (pa_s) pa_s[s] = per_atom_cutoff[a];
        if (ty_s) ty_s[s] = types[a];
    }

    visit_ctx c;
    for (int k = 0; k < 3; k++) {
        c.n[k] = g.n[k];
        c.nscan[k] = g.nscan[k];
        c.pbc[k] = pbc[k] ? 1 : 0;
        for (int m = 0; m < 3; m++) c.bin[k][m] = g.bin[k][m];
    }
    c.cutoff_sq = g.cutoff_sq;
    c.per_type_sq = per_type_cutoff_sq;
    c.ncutoffs = ncutoffs;
    c.raw = raw_s;
    c.rel = rel_s;
    c.pos = pos_s;
    c.per_atom = pa_s;
    c.types = ty_s;
    c.ukey = ukey;
    c.ufirst = ufirst;
    c.nu = nu;

    /* neighbour_list.cc:43-54: count pass, then prefix sum over original i. */
    int64_t *off = out->counts; /* counts[i+1] holds the count, then the scan */
    for (int32_t si = 0; si < nat; si++) {
        int64_t cnt = 0;
        visit(&c, si, emit_count, &cnt);
        off[sorted_atom[si] + 1] = cnt;
    }
    for (int32_t a = 0; a < nat; a++) off[a + 1] += off[a];
    const int64_t np = off[nat];
    out->npairs = np;

    /* neighbour_list.cc:56-94: exact-size outputs, fill pass. */
    if (np > 0) {
        if (quantities & Q_I) out->i = (int32_t *)malloc(sizeof(int32_t) * (size_t)np);
        if (quantities & Q_J) out->j = (int32_t *)malloc(sizeof(int32_t) * (size_t)np);
        if (quantities & Q_D) out->D = (double *)malloc(sizeof(double) * 3 * (size_t)np);
        if (quantities & Q_d) out->d = (double *)malloc(sizeof(double) * (size_t)np);
        if (quantities & Q_S) out->S = (int32_t *)malloc(sizeof(int32_t) * 3 * (size_t)np);
        for (int32_t si = 0; si < nat; si++) {
            fill_state f;
            f.i = sorted_atom[si];
            f.w = off[f.i];
            f.sorted_atom = sorted_atom;
            f.out = out;
            visit(&c, si, emit_fill, &f);
        }
    }

    free(raw);
    free(ka);
    free(ukey);
    free(ufirst);
    free(sorted_atom);
    free(raw_s);
    free(rel_s);
    free(pos_s);
    free(pa_s);
    free(ty_s);
    return ORACLE_OK;
}

/* ---- CSR helpers ---------------------------------------------------------- */

/* first_neighbours.cc:15-38. */
void oracle_first_neighbours(int32_t n, int64_t nn, const int32_t *i, int32_t *seed) {
    for (int64_t k = 0; k <= n; k++) seed[k] = -1;
    if (nn <= 0) {
        for (int64_t k = 0; k <= n; k++) seed[k] = 0;
        return;
    }
    seed[i[0]] = 0;
    for (int64_t k = 1; k < nn; k++) {
        if (i[k] != i[k - 1]) {
            for (int64_t l = (int64_t)i[k - 1] + 1; l <= i[k]; l++) seed[l] = (int32_t)k;
        }
    }
    for (int64_t k = (int64_t)i[nn - 1] + 1; k <= n; k++) seed[k] = (int32_t)nn;
}

/* triplet_list.cc:15-34: for each row r, every ordered pair (ij, ik) of its
   entries with ij != ik, both below the cutoff when distances are given. */
int64_t oracle_triplet_list(int32_t nfirst, const int32_t *first_i, const double *absdist,
                            double cutoff, int32_t *ij, int32_t *ik, int64_t cap) {
    int64_t t = 0;
    for (int32_t r = 0; r < nfirst - 1; r++) {
        for (int32_t a = first_i[r]; a < first_i[r + 1]; a++) {
            for (int32_t b = first_i[r]; b < first_i[r + 1]; b++) {
                if (a == b) continue;
                if (absdist && (absdist[a] >= cutoff || absdist[b] >= cutoff)) continue;
                if (ij && ik && t < cap) {
                    ij[t] = a;
                    ik[t] = b;
                }
                t++;
            }
        }
    }
    return t;
}
