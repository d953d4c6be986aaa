// nbl_stages.cuh -- the per-atom / per-cell bodies of the count phase's
// stages before the pair passes (binning, gather, work items, visit tables),
// shared by their own kernels (nbl_build.cu) and by the one-CTA count phase
// for small systems (nbl_small.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "nbl_build.cuh"
#include "nbl_internal.cuh"

namespace nbl {
namespace {

__device__ __forceinline__ int sys_of(const int64_t *__restrict__ bases, int nsys,
                                      int64_t a) {
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (bases[mid] <= a)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Open-addressing insert; returns the slot.  At most cap probes.
__device__ __forceinline__ uint32_t hash_insert(unsigned long long *hkey,
                                                unsigned long long mask,
                                                unsigned long long key, int *err) {
    unsigned long long h = mix64(key) & mask;
    for (unsigned long long p = 0; p <= mask; p++) {
        unsigned long long cur = *((volatile unsigned long long *)&hkey[h]);
        if (cur == key) return (uint32_t)h;
        if (cur == kHashEmpty) {
            unsigned long long prev = atomicCAS(&hkey[h], kHashEmpty, key);
            if (prev == kHashEmpty || prev == key) return (uint32_t)h;
        }
        h = (h + 1) & mask;
    }
    atomicOr(err, kErrInternal);
    return 0;
}


// Atom t (< natoms): its cell key and index for the sort.
__device__ __forceinline__ void bin_one(const BinArgs &a, int64_t t) {
    const int s = a.nsys > 1 ? sys_of(a.sys_atom_base, a.nsys, t) : 0;
    const SysDev &S = a.sys[s];
    double r[3] = {a.positions[3 * t + 0], a.positions[3 * t + 1],
                   a.positions[3 * t + 2]};
    int32_t raw[3];
    if (!raw_cell_of(S, r, raw)) atomicOr(a.err, kErrRange);
    int32_t c[3];
#pragma unroll
    for (int k = 0; k < 3; k++)
        c[k] = S.pbc[k] ? wrap_cell(raw[k], S.n[k]) : trunc_cell(raw[k], S.n[k]);
    const int64_t lin = (int64_t)c[0] + (int64_t)S.n[0] *
                                            ((int64_t)c[1] + (int64_t)S.n[1] * c[2]);
    uint32_t key;
    if (a.grid == kGridHashed) {
        const unsigned long long ck =
            ((unsigned long long)s << kHashSysShift) | (unsigned long long)lin;
        key = hash_insert(a.hkey, a.hmask, ck, a.err);
    } else if (a.grid == kGridMorton) {
        key = (uint32_t)(S.key_base + morton3(c[0], c[1], c[2]));
    } else {
        key = (uint32_t)(S.key_base + lin);
    }
    a.keys[t] = key;
    a.vals[t] = (int32_t)t;
}

// Sorted atom s (valid: s < natoms); every lane of the warp takes part (the
// per-system maxima and the occupied-cell list are aggregated per warp).
__device__ __forceinline__ void gather_one(const GatherArgs &a, int64_t s) {
    const bool valid = s < a.natoms;
    const unsigned full = 0xffffffffu;
    bool start = false;
    int sysid = 0;
    uint32_t tidx = 0;
    int32_t c[3] = {0, 0, 0};
    float amax = 0.f;
    if (valid) {
        const int32_t at = a.vals[s];
        sysid = a.nsys > 1 ? sys_of(a.sys_atom_base, a.nsys, at) : 0;
        const SysDev &S = a.sys[sysid];
        const double r[3] = {a.positions[3 * (int64_t)at + 0],
                             a.positions[3 * (int64_t)at + 1],
                             a.positions[3 * (int64_t)at + 2]};
        int32_t raw[3];
        raw_cell_of(S, r, raw);  // range errors were flagged by k_bin
        int32_t rc[3], q[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            if (S.pbc[k]) {
                c[k] = wrap_cell(raw[k], S.n[k]);
                rc[k] = raw[k];
                q[k] = floor_div(raw[k], S.n[k]);
            } else {
                c[k] = trunc_cell(raw[k], S.n[k]);
                rc[k] = c[k];
                q[k] = (raw[k] - c[k]) / S.n[k];  // C truncating division
            }
        }
        // neighbour_list.cc:157-159: ((r - r1 b1) - r2 b2) - r3 b3
        double rel[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double v = dsub(r[k], dmul((double)rc[0], S.bin[0][k]));
            v = dsub(v, dmul((double)rc[1], S.bin[1][k]));
            v = dsub(v, dmul((double)rc[2], S.bin[2][k]));
            rel[k] = v;
        }
        double w64 = 0.0;
        float w32 = 0.f;
        if (S.cutoff_kind == kCutPerAtom) {
            w64 = a.per_atom[at];
            w32 = __double2float_rn(w64);
        } else if (S.cutoff_kind == kCutPerType) {
            w32 = __int_as_float(a.types[at]);
        }
        a.pos64[s] = make_double4(rel[0], rel[1], rel[2], w64);
        a.pos32[s] = make_float4(__double2float_rn(rel[0]), __double2float_rn(rel[1]),
                                 __double2float_rn(rel[2]), w32);
        a.aux[s] = make_int4(at, q[0], q[1], q[2]);
        amax = __double2float_ru(fmax(fabs(rel[0]), fmax(fabs(rel[1]), fabs(rel[2]))));

        const uint32_t key = a.keys[s];
        const int64_t lin = (int64_t)c[0] +
                            (int64_t)S.n[0] * ((int64_t)c[1] + (int64_t)S.n[1] * c[2]);
        tidx = (a.grid == kGridMorton) ? (uint32_t)(S.cell_base + lin) : key;
        start = (s == 0) || (a.keys[s - 1] != key);
        const bool end = (s == a.natoms - 1) || (a.keys[s + 1] != key);
        if (start) a.table[tidx].x = (int32_t)s;
        if (end) a.table[tidx].y = (int32_t)(s + 1);
    }
    // Per-system max |rel| (non-negative floats order like their bit patterns):
    // one atomic per warp when the warp lies inside one system, else per lane.
    {
        const int lane = threadIdx.x & 31;
        const int s0 = __shfl_sync(full, sysid, 0);
        const bool uni = __all_sync(full, !valid || sysid == s0);
        const unsigned bits = valid ? (unsigned)__float_as_int(amax) : 0u;
        if (uni) {
            const unsigned mx = __reduce_max_sync(full, bits);
            const unsigned anyv = __ballot_sync(full, valid);
            if (lane == 0 && anyv) atomicMax(reinterpret_cast<unsigned *>(a.amax) + s0, mx);
        } else if (valid) {
            atomicMax(reinterpret_cast<unsigned *>(a.amax) + sysid, bits);
        }
    }
    // Occupied-cell work list (warp-aggregated append).
    const unsigned m = __ballot_sync(full, start);
    if (m) {
        const int lane = threadIdx.x & 31;
        int base = 0;
        if (lane == __ffs(m) - 1) base = atomicAdd(a.n_home, __popc(m));
        base = __shfl_sync(full, base, __ffs(m) - 1);
        if (start) {
            HomeCell h;
            h.tidx = (int32_t)tidx;
            h.sys = sysid;
            h.c[0] = c[0];
            h.c[1] = c[1];
            h.c[2] = c[2];
            h.pad = 0;
            a.home[base + __popc(m & lanemask_lt())] = h;
        }
    }
}

// Run length R of the tile builder: max_run, or (max_run == 0) 1 at six or
// more atoms per occupied cell, else about itile / (2 x occupancy); at most
// kMaxRun.
__device__ __forceinline__ int tiles_run_length(int nh, int64_t natoms, int itile,
                                                int max_run) {
    int R = max_run;
    if (R == 0) {
        const float occ = (float)natoms / (float)max(nh, 1);
        R = occ >= 6.f ? 1 : min(kMaxRun, max(1, (int)((float)itile / (2.f * occ))));
    }
    return min(R, kMaxRun);
}

// Occupied cell h (h < nh valid) -> its work items; every lane of the warp
// takes part (one atomic per warp reserves the warp's items).
// (No __restrict__ here: the one-CTA count phase calls this on cells and
// slices it wrote itself earlier in the same kernel.)
__device__ __forceinline__ void tiles_one(const HomeCell *home, const int2 *table,
                                          const SysDev *sys, WorkItem *items, int *n_items,
                                          int itile, int R, int h, int nh) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int2 hs = make_int2(0, 0);
    HomeCell hc{};
    if (h < nh) {
        hc = home[h];
        hs = table[hc.tidx];
    }
    int nt = (hs.y - hs.x + itile - 1) / itile;
    int run = 1, run_atoms = 0;
    if (R > 1 && h < nh) {
        const SysDev &S = sys[hc.sys];
        if (S.nscan[0] == 1 && S.nscan[1] == 1 && S.nscan[2] == 1) {
            const int x = hc.c[0];
            const int xb = (x / R) * R, xe = min(xb + R, S.n[0]);
            int total = 0, first = -1, last = -1;
            for (int xc = xb; xc < xe; xc++) {
                const int2 sl = table[hc.tidx + (xc - x)];
                const int n = sl.y - sl.x;
                if (n > 0) {
                    total += n;
                    if (first < 0) first = xc;
                    last = xc;
                }
            }
            if (total <= itile && first != last) {  // two or more occupied cells
                nt = (x == first) ? 1 : 0;
                run = last - first + 1;
                run_atoms = total;
            }
        }
    }
    int incl = nt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int o = __shfl_up_sync(full, incl, d);
        if (lane >= d) incl += o;
    }
    const int tot = __shfl_sync(full, incl, 31);
    int first = 0;
    if (lane == 0 && tot > 0) first = atomicAdd(n_items, tot);
    first = __shfl_sync(full, first, 0) + incl - nt;
    for (int t = 0; t < nt; t++) {
        WorkItem w;
        w.c[0] = hc.c[0];
        w.c[1] = hc.c[1];
        w.c[2] = hc.c[2];
        w.sys = hc.sys;
        w.ib = hs.x + itile * t;
        w.nt = run > 1 ? run_atoms : min(itile, hs.y - w.ib);
        w.tidx = hc.tidx;
        w.run = run;
        items[first + t] = w;
    }
}

// The visited offsets of system S (its visit table, if it has one), in the
// traversal's z/y/x order, spread over `nthr` threads.
__device__ __forceinline__ void visit_fill(const SysDev &S, VisitDev *__restrict__ visit,
                                           int tid, int nthr) {
    if (S.visit_base < 0) return;
    const int nx = S.nscan[0], ny = S.nscan[1], nz = S.nscan[2];
    const int wx = 2 * nx + 1, wy = 2 * ny + 1;
    for (int v = tid; v < S.nvisit; v += nthr) {
        const int xr = v % wx, rest = v / wx;
        const int yr = rest % wy, zr = rest / wy;
        const int d[3] = {xr - nx, yr - ny, zr - nz};
        double o[3];
        visit_offset(S, d, o);
        VisitDev e;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            e.off[k] = o[k];
            e.off32[k] = __double2float_rn(o[k]);
            e.d[k] = d[k];
        }
        visit[S.visit_base + v] = e;
    }
}

}  // namespace
}  // namespace nbl
