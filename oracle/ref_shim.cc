/*
 * ref_shim.cc -- TEST INFRASTRUCTURE ONLY.
 *
 * A C-ABI shim over the reference's own C++ CPU core, so the oracle tests and
 * the CPU-baseline leg of bench.py can call the unmodified reference code
 * (src/libneighbours/neighbour_list.cc:99 `matscipy::neighbour_list`) through
 * ctypes.  oracle/Makefile compiles this file together with the reference
 * sources where they lie (nothing is copied) into oracle/_ref/.
 *
 * The copy of each requested quantity into caller-owned flat buffers mirrors
 * what the reference's Python binding does after the core call
 * (language_bindings/python/bind_py_neighbours.cc:37-75, 222-237).
 */
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "error.hh"
#include "first_neighbours.hh"
#include "neighbour_list.hh"
#include "triplet_list.hh"

using namespace matscipy;

template <typename T>
static T *dup(const std::vector<T> &v) {
    if (v.empty()) return nullptr;
    T *p = static_cast<T *>(std::malloc(v.size() * sizeof(T)));
    std::memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

extern "C" {

typedef struct {
    int64_t npairs;
    int32_t *i;
    int32_t *j;
    double *D;
    double *d;
    int32_t *S;
} ref_result_t;

int ref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

const char *ref_last_error(void) { return error_string; }

/* Same arguments as the core (neighbour_list.hh:63-69), pbc as int[3]. */
int ref_neighbour_list(int quantities, const double *origin, const double *cell,
                       const double *inv_cell, const int *pbc_i, int nat,
                       const double *r, double cutoff, const double *per_atom,
                       const double *per_type_sq, int ncutoffs,
                       const int *types, int morton, ref_result_t *out) {
    bool pbc[3] = {pbc_i[0] != 0, pbc_i[1] != 0, pbc_i[2] != 0};
    NeighbourList nl;
    error_t e = neighbour_list(quantities, origin, cell, inv_cell, pbc, nat, r,
                               cutoff, per_atom, per_type_sq, ncutoffs, types,
                               nl, morton ? CellOrder::Morton : CellOrder::Linear);
    std::memset(out, 0, sizeof(*out));
    if (e != NL_SUCCESS) return 1;
    out->npairs = nl.npairs;
    out->i = dup(nl.first);
    out->j = dup(nl.secnd);
    out->D = dup(nl.distvec);
    out->d = dup(nl.absdist);
    out->S = dup(nl.shift);
    return 0;
}

/* first_neighbours (first_neighbours.hh) on the reference's own code. */
void ref_first_neighbours(int n, int nn, const int *i, int *seed) {
    first_neighbours(n, nn, i, seed);
}

/* triplet_list (triplet_list.hh); returns the count, copies at most cap. */
int64_t ref_triplet_list(int nfirst, const int *first_i, const double *absdist,
                         double cutoff, int *ij, int *ik, int64_t cap) {
    std::vector<index_t> a, b;
    triplet_list(nfirst, first_i, absdist, cutoff, a, b);
    const int64_t t = (int64_t)a.size();
    if (ij && ik) {
        for (int64_t k = 0; k < t && k < cap; k++) {
            ij[k] = a[k];
            ik[k] = b[k];
        }
    }
    return t;
}

void ref_result_free(ref_result_t *o) {
    std::free(o->i);
    std::free(o->j);
    std::free(o->D);
    std::free(o->d);
    std::free(o->S);
    std::memset(o, 0, sizeof(*o));
}

}  // extern "C"
