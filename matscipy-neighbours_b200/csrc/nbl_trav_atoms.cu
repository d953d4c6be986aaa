// nbl_trav_atoms.cu -- the pair passes with one thread per atom, for sparse
// grids.
//
// On a grid with about one or two atoms per occupied cell (a slab or a
// cluster in a large vacuum box) a work item of the warp passes holds a
// couple of atoms, so a warp spends its set-up (segments, staging, hit
// words, position table) on a handful of pairs.  Here each thread takes one
// sorted atom and walks its visited cells itself, in the reference's z/y/x
// order (the system's visit table) and each cell's slice in ascending atom
// order, with the reference's exact FP64 test (neighbour_visit.hh:88-109):
// the count pass stores the atom's row length, the fill pass writes the row
// at offsets[i] in the same order (neighbour_list.cc:69-94).  The output is
// the warp passes' output, bit for bit.  Neighbouring threads hold atoms of
// the same or adjacent cells (the atoms are cell-sorted), so their visits
// read the same table entries and candidates.
#include "nbl_stages.cuh"
#include "nbl_traverse.cuh"

namespace nbl {
namespace {

constexpr int kAtomThreads = 128;

// Inverse of spread3: the low 10-bit coordinate interleaved at every third bit.
__device__ __forceinline__ uint32_t compact3(uint32_t x) {
    x &= 0x09249249u;
    x = (x | (x >> 2)) & 0x030c30c3u;
    x = (x | (x >> 4)) & 0x0300f00fu;
    x = (x | (x >> 8)) & 0x030000ffu;
    x = (x | (x >> 16)) & 0x000003ffu;
    return x;
}

// System and folded home-cell coordinates of sorted atom si (batch atom
// `at`), from its sorted cell key.  False (and kErrInternal) if the key does
// not name a cell of the grid, which only a failed hash insert (already
// flagged) can cause: the atom is then skipped.
__device__ __forceinline__ bool atom_home(const TraverseArgs &a, int64_t si, int at, int &sys,
                                          int32_t c[3]) {
    const uint32_t key = a.skeys[si];
    int64_t lin;
    if (a.grid == kGridHashed) {
        const unsigned long long hk =
            (unsigned long long)key <= a.hmask ? a.hkey[key] : kHashEmpty;
        sys = (int)(hk >> kHashSysShift);
        lin = (int64_t)(hk & ((1ull << kHashSysShift) - 1));
        if (hk == kHashEmpty || sys >= a.nsys) {
            atomicOr(a.err, kErrInternal);
            return false;
        }
    } else {
        sys = a.nsys > 1 ? sys_of(a.sys_atom_base, a.nsys, at) : 0;
        const SysDev &S = a.sys[sys];
        const uint32_t k = key - (uint32_t)S.key_base;
        if (a.grid == kGridMorton) {
            c[0] = (int32_t)compact3(k);
            c[1] = (int32_t)compact3(k >> 1);
            c[2] = (int32_t)compact3(k >> 2);
        } else {
            lin = (int64_t)k;
        }
    }
    const SysDev &S = a.sys[sys];
    if (a.grid != kGridMorton) {
        const int64_t nxy = (int64_t)S.n[0] * S.n[1];
        c[2] = (int32_t)(lin / nxy);
        const int64_t r = lin - (int64_t)c[2] * nxy;
        c[1] = (int32_t)(r / S.n[0]);
        c[0] = (int32_t)(r - (int64_t)c[1] * S.n[0]);
    }
    if (c[0] < 0 || c[0] >= S.n[0] || c[1] < 0 || c[1] >= S.n[1] || c[2] < 0 ||
        c[2] >= S.n[2]) {
        atomicOr(a.err, kErrInternal);
        return false;
    }
    return true;
}

// Neighbour cell of home cell c at cell offset d: folded coordinates and
// image counts (periodic axes), false when it lies outside an open axis
// (neighbour_visit.hh:63-84; the same folding as the warp passes).
__device__ __forceinline__ bool visit_cell(const SysDev &S, const int32_t c[3],
                                           const int32_t d[3], int32_t cj[3], int32_t m[3]) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        int32_t x = c[k] + d[k];
        m[k] = 0;
        if (S.pbc[k]) {
            const int32_t n = S.n[k];
            if (x < 0 && x >= -n) {
                m[k] = -1;
                x += n;
            } else if (x >= n && x < 2 * n) {
                m[k] = 1;
                x -= n;
            } else if (x < 0 || x >= n) {
                m[k] = floor_div(x, n);
                x -= m[k] * n;
            }
        } else if (x < 0 || x >= S.n[k]) {
            return false;
        }
        cj[k] = x;
    }
    return true;
}

// One pair of the row (FILL): exact FP64 D, d and S at slot s, or its matrix
// entry (rank s - row0 < mat_k).
template <bool ALL5>
__device__ __forceinline__ void emit_pair(const TraverseArgs &a, const Hot &H, const int4 &ai,
                                          const double4 &pi, const double4 &pj, int32_t sj,
                                          const double *off, const int32_t m[3], long long s,
                                          long long row0) {
    const double dx = dadd(dsub(pj.x, pi.x), off[0]);
    const double dy = dadd(dsub(pj.y, pi.y), off[1]);
    const double dz = dadd(dsub(pj.z, pi.z), off[2]);
    const int4 aj = a.aux[sj];
    const int32_t jl = (int32_t)(aj.x - H.atom_base);
    if (!ALL5 && a.mat_k > 0) {
        const long long rank = s - row0;
        if (rank < a.mat_k) {
            const long long q = (long long)ai.x * a.mat_k + rank;
            a.mat_idx[q] = jl;
            a.mat_dist[3 * q + 0] = dx;
            a.mat_dist[3 * q + 1] = dy;
            a.mat_dist[3 * q + 2] = dz;
        }
        return;
    }
    if (s >= a.capacity) {
        atomicOr(a.err, kErrCapacity);
        return;
    }
    if (ALL5 || a.first) __stcs(a.first + s, (int32_t)(ai.x - H.atom_base));
    if (ALL5 || a.second) __stcs(a.second + s, jl);
    if (ALL5 || a.absdist) {
        const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
        __stcs(a.absdist + s, __dsqrt_rn(r2));
    }
    if (ALL5 || a.distvec) {
        double *D = a.distvec + 3 * s;
        __stcs(D, dx);
        __stcs(D + 1, dy);
        __stcs(D + 2, dz);
    }
    if (ALL5 || a.shift) {
        int32_t *Sv = a.shift + 3 * s;
        __stcs(Sv, ai.y - ((H.pbc_bits & 1) ? aj.y : 0) + m[0]);
        __stcs(Sv + 1, ai.z - ((H.pbc_bits & 2) ? aj.z : 0) + m[1]);
        __stcs(Sv + 2, ai.w - ((H.pbc_bits & 4) ? aj.w : 0) + m[2]);
    }
}

// One sorted atom's row: its length (FILL = false, into counts) or its pairs
// (FILL = true, at offsets[i] on).  ALL5: all five outputs, no matrix.
template <int KIND, bool FILL, bool ALL5>
__device__ __forceinline__ void atom_row(const TraverseArgs &a, int64_t si) {
    const int4 ai = a.aux[si];
    if (checked_fail(ai.x < 0 || ai.x >= a.natoms, a.err)) return;
    if (ai.x < a.i_lo || ai.x >= a.i_hi) return;
    int sys = 0;
    int32_t cc[3] = {0, 0, 0};
    if (!atom_home(a, si, ai.x, sys, cc)) return;
    const SysDev &S = a.sys[sys];
    Hot H;
    H.lo_rc = H.hi_rc = H.band = 0.f;
    H.cutoff_sq = S.cutoff_sq;
    H.pbc_bits = (S.pbc[0] ? 1 : 0) | (S.pbc[1] ? 2 : 0) | (S.pbc[2] ? 4 : 0);
    H.ncut = S.ncutoffs;
    H.pt_base = S.pt_base;
    H.vrun = -1;
    H.atom_base = S.atom_base;
    const double4 pi = a.pos64[si];
    const float wi = a.pos32[si].w;
    long long row0 = 0, slot = 0;
    if (FILL) {
        row0 = (long long)a.offsets[ai.x];
        slot = row0;
    }
    int cnt = 0;
    const VisitDev *vt = a.visit + S.visit_base;
    const int nv = S.nvisit;
    for (int v = 0; v < nv; v++) {
        const VisitDev &e = vt[v];
        const int32_t d[3] = {e.d[0], e.d[1], e.d[2]};
        int32_t cj[3], m[3];
        if (!visit_cell(S, cc, d, cj, m)) continue;
        const int2 sl = cell_lookup(a, S, sys, cj[0], cj[1], cj[2]);
        if (checked_fail(sl.x < 0 || sl.y < sl.x || (long long)sl.y > a.natoms, a.err))
            continue;
        // the atom itself (zero offset) is skipped
        const int32_t self = (d[0] == 0 && d[1] == 0 && d[2] == 0) ? (int32_t)si : -1;
        for (int32_t sj = sl.x; sj < sl.y; sj++) {
            if (sj == self) continue;
            const double4 pj = a.pos64[sj];
            const float tj = KIND == kCutPerType ? a.pos32[sj].w : 0.f;
            if (!exact_inside<KIND>(H, a, pi, pj, e.off, wi, tj)) continue;
            if (FILL)
                emit_pair<ALL5>(a, H, ai, pi, pj, sj, e.off, m, slot++, row0);
            else
                cnt++;
        }
    }
    if (!FILL) {
        a.counts[ai.x] = cnt;
        return;
    }
    // the row must end exactly where the next one starts; matrix row lengths
    const long long end = (long long)a.offsets[ai.x + 1];
    if (slot != end) atomicOr(a.err, kErrInternal);
    if (!ALL5 && a.mat_k > 0) {
        const long long deg = end - row0;
        a.mat_count[ai.x] = (int32_t)deg;
        if (deg > a.mat_k) atomicOr(a.mat_overflow, 1);
    }
}

template <int KIND, bool FILL, bool ALL5>
__global__ void __launch_bounds__(kAtomThreads)
k_atoms(TraverseArgs a) {
    const int64_t si = (int64_t)blockIdx.x * kAtomThreads + threadIdx.x;
    if (si < a.natoms) atom_row<KIND, FILL, ALL5>(a, si);
}

template <bool FILL, bool ALL5>
TravKernel atoms_kernel(int kind) {
    if (kind == kCutPerAtom) return k_atoms<kCutPerAtom, FILL, ALL5>;
    if (kind == kCutPerType) return k_atoms<kCutPerType, FILL, ALL5>;
    return k_atoms<kCutScalar, FILL, ALL5>;
}

cudaError_t launch_atoms(TravKernel k, const TraverseArgs &a, cudaStream_t st) {
    if (a.natoms <= 0) return cudaSuccess;
    if (a.visit == nullptr || a.skeys == nullptr) return cudaErrorInvalidValue;
    const int64_t grid = (a.natoms + kAtomThreads - 1) / kAtomThreads;
    k<<<(unsigned)grid, kAtomThreads, 0, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_count_atoms(int kind, const TraverseArgs &a, cudaStream_t st) {
    return launch_atoms(atoms_kernel<false, false>(kind), a, st);
}

cudaError_t launch_fill_atoms(int kind, const TraverseArgs &a, cudaStream_t st) {
    const bool all5 = a.first && a.second && a.distvec && a.absdist && a.shift && a.mat_k == 0;
    return launch_atoms(all5 ? atoms_kernel<true, true>(kind) : atoms_kernel<true, false>(kind),
                        a, st);
}

}  // namespace nbl
