// nbl_internal.cuh -- shared device/host definitions of the B200 engine.
//
// Data layout in HBM (one "batch" = one or more independent systems whose
// atoms are concatenated; a single neighbour_list call is a batch of one):
//
//   SysDev[nsys]        per-system grid definition (host-planned, bit-exact)
//   keys/vals[N]        radix-sort keys (cell key) and global atom indices
//   table[ncells]       int2 {first, end} slice of each cell in sorted order
//                       (dense: indexed by cell_base + linear cell; hashed:
//                       indexed by hash slot)
//   hkey[cap]           hashed grid only: composite (system, linear cell) key
//   pos64[N]  double4   cell-sorted bin-relative position (x, y, z) and the
//                       per-atom cutoff radius (w) -- the FP64 operands
//   pos32[N]  float4    the same position rounded to FP32 (x, y, z) and the
//                       per-atom radius (FP32) or the type id (int bits) (w)
//   aux[N]    int4      (global atom index, q0, q1, q2): q is the atom's
//                       periodic image index (periodic axes) or the
//                       reference's shift quirk (non-periodic axes)
//   home[N]   HomeCell  occupied cells (the work items of the pair kernels)
//   counts[N] int32     neighbours per atom (original order)
//   offsets[N+1] int64  exclusive prefix of counts = row starts
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace nbl {

constexpr int kGridDense = 1;
constexpr int kGridMorton = 2;
constexpr int kGridHashed = 3;

constexpr int kCutScalar = 0;
constexpr int kCutPerAtom = 1;
constexpr int kCutPerType = 2;

// Device error bits (accumulated with atomicOr, read back by the host).
constexpr int kErrRange = 1;      // non-finite or out-of-range position
constexpr int kErrCapacity = 2;   // output slot beyond capacity
constexpr int kErrInternal = 4;   // a device-side bound was hit

// Checked build (-DNBL_CHECKED=1, libnbl_b200_checked.so): the traversal
// kernels also test the indices that the release build holds in bounds by
// construction -- every cell slice within [0, natoms], every candidate and
// home atom below natoms, every hit word below the pool size, and every
// output slot inside its own row [offsets[i], offsets[i+1]).  A failed test
// sets kErrInternal and skips the access; it never traps.
#ifndef NBL_CHECKED
#define NBL_CHECKED 0
#endif
constexpr bool kChecked = NBL_CHECKED != 0;

// True (and kErrInternal recorded) when a checked build sees `bad`.
__device__ __forceinline__ bool checked_fail(bool bad, int *err) {
    if constexpr (kChecked) {
        if (bad) {
            atomicOr(err, kErrInternal);
            return true;
        }
    }
    return false;
}

// Composite key layout of the hashed grid: system id above bit 43.
constexpr int kHashSysShift = 43;
constexpr unsigned long long kHashEmpty = ~0ull;

// Per-system grid definition.  Everything here is computed on the host with
// the reference's operation order (cell_list.cc:153-182,
// neighbour_list.cc:169-192) so device arithmetic that consumes it is
// bit-identical to the reference CPU path.
struct SysDev {
    double origin[3];
    double inv[9];       // row-major inv(cell.T)
    double bin[3][3];    // bin[k][c] = cell[k][c] / n[k]
    double cutoff;       // binning / global cutoff
    double cutoff_sq;    // cutoff * cutoff (FP64, as the reference)
    double off_max;      // bound on |offset component| over visited offsets
    int32_t n[3];        // cells per lattice direction
    int32_t nscan[3];    // cells scanned each way (NeighbourContext nx/ny/nz)
    int32_t pbc[3];
    int32_t nat;
    int64_t atom_base;   // first atom of this system in the batch arrays
    int64_t cell_base;   // dense: first table entry of this system
    int64_t key_base;    // sort-key base (dense: == cell_base; Morton: own)
    int32_t cutoff_kind; // kCutScalar / kCutPerAtom / kCutPerType
    int32_t ncutoffs;
    int32_t pt_base;     // first entry of this system's per-type tables
    int32_t nvisit;      // (2nx+1)(2ny+1)(2nz+1)
    int64_t visit_base;  // first VisitDev entry of this system, -1: computed per item
};

// One visited neighbour offset of a system (neighbour_visit.hh:63-84): the
// cell offset, the offset vector in FP64 (the reference's operation order)
// and its FP32 rounding, computed once per call by the count phase's init.
struct VisitDev {
    double off[3];
    float off32[3];
    int32_t d[3];
};

struct HomeCell {
    int32_t tidx;  // table index of the cell
    int32_t sys;
    int32_t c[3];  // folded cell coordinates
    int32_t pad;
};

// One work item of the pair passes, self-contained so that a warp needs one
// 32-byte load to start it: the home cell (folded coordinates, system) and
// the tile of its sorted atoms [ib, ib + nt).  A run (run > 1, dense grid
// only) is `run` consecutive home cells along x starting at c, whose atoms
// (contiguous in sorted order) form one tile; their neighbour cells are
// visited once for the whole run.
struct __align__(16) WorkItem {
    int32_t c[3];
    int32_t sys;
    int32_t ib;
    int32_t nt;
    int32_t tidx;  // table index of the (first) home cell
    int32_t run;   // home cells in the item (1: a single cell)
};

// Home cells per run at most (and the bound on a run's x extent the FP32
// guard band is sized for).
constexpr int kMaxRun = 8;

// Mask-pool reference of one (work item, segment batch), as the count stores
// it: the first word in the low 40 bits, the batch's 32-candidate chunks per
// atom above them; -1 when the item's words are not in the pool.
constexpr int kMaskBaseBits = 40;
__host__ __device__ __forceinline__ long long mask_ref(long long base, int nchunks) {
    return base | ((long long)nchunks << kMaskBaseBits);
}
__host__ __device__ __forceinline__ long long mask_ref_base(long long ref) {
    return ref < 0 ? -1ll : (ref & ((1ll << kMaskBaseBits) - 1));
}
__host__ __device__ __forceinline__ int mask_ref_chunks(long long ref) {
    return ref < 0 ? 0 : (int)(ref >> kMaskBaseBits);
}

// Asynchronous global -> shared copies (cp.async, sm_80 and later): the data
// lands in shared memory while the warp goes on; cp_async_wait waits for all
// of the calling thread's copies (then __syncwarp before other lanes read).
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Kernel launches issued by the calling host thread (reported through
// nbl_launch_count()); every launch site bumps it.
void count_launch(int n = 1);

// ---- bit-exact FP64 helpers (no contraction into FMA anywhere) ------------

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// Periodic wrap of a cell coordinate into [0, n) (tools.hh:43-46), by modulo.
__host__ __device__ __forceinline__ int32_t wrap_cell(int32_t i, int32_t n) {
    int32_t r = i % n;
    return r < 0 ? r + n : r;
}
// Non-periodic clamp into [0, n) (tools.hh:49-56).
__host__ __device__ __forceinline__ int32_t trunc_cell(int32_t i, int32_t n) {
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}
// Floor division for the periodic image index.
__host__ __device__ __forceinline__ int32_t floor_div(int32_t a, int32_t n) {
    int32_t q = a / n;
    return (a % n != 0 && ((a < 0) != (n < 0))) ? q - 1 : q;
}

// Raw (un-wrapped) cell coordinates of one atom: tools.hh:55-67 with
// mat_mul_vec (tools.hh:35-41): s_k = ((0 + m_k0 d0) + m_k1 d1) + m_k2 d2,
// raw_k = (int) floor(s_k * n_k).  Returns false when a coordinate is not
// finite or lies more than 2^29 cells away (the reference's int arithmetic on
// such values is undefined).
__device__ __forceinline__ bool raw_cell_of(const SysDev &S, const double *r,
                                            int32_t raw[3]) {
    double d0 = dsub(r[0], S.origin[0]);
    double d1 = dsub(r[1], S.origin[1]);
    double d2 = dsub(r[2], S.origin[2]);
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        double s = 0.0;
        s = dadd(s, dmul(S.inv[3 * k + 0], d0));
        s = dadd(s, dmul(S.inv[3 * k + 1], d1));
        s = dadd(s, dmul(S.inv[3 * k + 2], d2));
        double f = floor(dmul(s, (double)S.n[k]));
        bool in = (f > -536870912.0) && (f < 536870912.0);
        ok = ok && in;
        raw[k] = in ? (int32_t)f : 0;
    }
    return ok;
}

// Offset vector of cell offset d (neighbour_visit.hh:67,73,80):
// off3 = z b3; off2 = off3 + y b2; off = off2 + x b1, in FP64 without FMA.
__device__ __forceinline__ void visit_offset(const SysDev &S, const int d[3], double o[3]) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        double v = dmul((double)d[2], S.bin[2][k]);
        v = dadd(v, dmul((double)d[1], S.bin[1][k]));
        v = dadd(v, dmul((double)d[0], S.bin[0][k]));
        o[k] = v;
    }
}

// 64-bit mixer for the hashed grid (splitmix64 finaliser).
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

// Lanes below the calling lane.
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Slice of hashed cell `key`: open addressing with linear probing, at most
// mask + 1 probes; an absent key gives an empty slice, a full table without
// the key sets kErrInternal (never a wait).
__device__ __forceinline__ int2 hash_find(const unsigned long long *__restrict__ hkey,
                                          unsigned long long mask,
                                          const int2 *__restrict__ table,
                                          unsigned long long key, int *err) {
    unsigned long long h = mix64(key) & mask;
    for (unsigned long long p = 0; p <= mask; p++) {
        unsigned long long cur = hkey[h];
        if (cur == key) return table[h];
        if (cur == kHashEmpty) return make_int2(0, 0);
        h = (h + 1) & mask;
    }
    atomicOr(err, kErrInternal);
    return make_int2(0, 0);
}

// Interleave the low 10 bits of three coordinates (Morton / Z-order key).
__host__ __device__ __forceinline__ uint32_t spread3(uint32_t x) {
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}
__host__ __device__ __forceinline__ uint32_t morton3(int32_t a, int32_t b, int32_t c) {
    return spread3((uint32_t)a) | (spread3((uint32_t)b) << 1) |
           (spread3((uint32_t)c) << 2);
}

// ---- FP32 guard band ---------------------------------------------------------
//
// The FP32 filter computes dr' = fl32(c - a) with c = fl32(fl32(rel_j) +
// fl32(off)) staged per candidate and a = fl32(rel_i), then
// r2' = fl32(fma(dz, dz, fma(dy, dy, dx * dx))).  With u = 2^-24,
// A = max |rel component| over the system's atoms, C = max |offset component|
// and M = 2A + C, each component error is |dr'_k - dr_k| <= 3.01 u M, and for
// any pair whose exact r2 lies below a threshold T <= R^2 (R = binning
// cutoff), |r2' - r2| <= 18.1 u M R + 27.3 u^2 M^2 + 3.01 u R^2.  The FP32
// threshold (rc^2, (r_i + r_j)^2 in FP32, or the per-type square rounded to
// FP32) is within 6.1 u R^2 of the FP64 one, and the reference's own FP64 r2
// differs from the exact value by less than 2^-50 M R.  The band
//     B = 48 u (M R + R^2) + 64 u^2 M^2
// therefore exceeds the total error by a factor of at least 2.3, so
// r2' < T' - B implies the reference accepts the pair and r2' >= T' + B
// implies it rejects it; only candidates in between are re-tested with the
// reference's exact FP64 arithmetic.
__host__ __device__ __forceinline__ double guard_band(double M, double R) {
    const double u = 5.9604644775390625e-08;  // 2^-24
    return 48.0 * u * (M * R + R * R) + 64.0 * u * u * M * M;
}

}  // namespace nbl
