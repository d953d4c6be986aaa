// nbl_build.cu -- the neighbour-list kernels for sm_100a.
//
// Pipeline (one launch sequence per batch of systems, all on one stream):
//   k_bin       per atom: raw cell (reference arithmetic), fold, cell key;
//               hashed grid: insert the cell into the open-addressing table
//   radix sort  (nbl_sort.cu) stable by cell key -> cell-sorted atom order
//   k_gather    per sorted atom: bin-relative position (FP64, reference
//               arithmetic), its FP32 copy, image indices, cell slices,
//               occupied-cell work list
//   k_traverse<COUNT>  per occupied home cell: neighbour counts per atom
//   scan        (nbl_sort.cu) counts -> row offsets, total pair count
//   k_traverse<FILL>   per occupied home cell: writes i, j, D, d, S
//
// The traversal reproduces neighbour_visit.hh:51-120 exactly: the same
// visited offsets in the same z/y/x order, the same cell slices in ascending
// atom order, the same FP64 operations (no FMA contraction: every FP64 op is an
// explicit __d*_rn intrinsic), so the output is the reference CPU output,
// including the order of pairs within a row.
//
// Work decomposition (instead of the reference's thread-per-atom loop): one
// CTA per occupied home cell.  The CTA enumerates the visited neighbour cells
// ("segments"), stages their atoms ("candidates") in shared memory, and each
// warp takes one atom i of the home cell and sweeps the candidates 32 at a
// time: FP32 distance filter (or plain FP64), __ballot_sync + __popc for the
// count, and in the fill pass the hits go into a per-warp queue that is
// drained 32 pairs at a time so that the FP64 epilogue and the stores run
// with full warps and near-contiguous addresses.
#include <cstdint>
#include <type_traits>

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

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
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

}  // namespace

// ---------------------------------------------------------------------------
// k_bin
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_bin(BinArgs a) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.natoms) return;
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

// ---------------------------------------------------------------------------
// k_gather
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_gather(GatherArgs a) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
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

// ---------------------------------------------------------------------------
// k_traverse: the count and fill passes
// ---------------------------------------------------------------------------
namespace {

constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;
constexpr int kSegBatch = 128;
constexpr int kITile = 64;
constexpr int kQueue = 64;

template <bool FP32>
struct TileCfg {
    static constexpr int kCand = FP32 ? 1024 : 512;
};

template <bool FP32>
struct __align__(16) TravSmem {
    // segments (visited neighbour cells) of the current batch
    double seg_off[kSegBatch][3];
    int32_t seg_m[kSegBatch][3];
    int32_t seg_b[kSegBatch];
    int32_t seg_pref[kSegBatch + 1];
    uint8_t seg_zero[kSegBatch];
    // candidates of the current tile
    typename std::conditional<FP32, float4, double4>::type cand[TileCfg<FP32>::kCand];
    int32_t cand_sj[TileCfg<FP32>::kCand];
    uint8_t cand_seg[TileCfg<FP32>::kCand];
    // atoms i of the current i-tile
    double4 i64[kITile];
    float4 i32[kITile];
    int4 iaux[kITile];
    long long istate[kITile];  // count (COUNT) or write cursor (FILL)
    long long istart[kITile];  // row start (FILL)
    // per-warp emit queue (FILL)
    int32_t q[kWarps][kQueue];
    long long qw[kWarps][kQueue];
    int32_t scan_warp[33];
    SysDev sys;
};

struct Thresh {
    float lo_rc, hi_rc, band;
};

__device__ __forceinline__ int2 cell_lookup(const TraverseArgs &a, const SysDev &S,
                                            int sysid, int32_t c0, int32_t c1,
                                            int32_t c2) {
    const int64_t lin = (int64_t)c0 + (int64_t)S.n[0] *
                                          ((int64_t)c1 + (int64_t)S.n[1] * c2);
    if (a.grid != kGridHashed) return a.table[S.cell_base + lin];
    const unsigned long long key =
        ((unsigned long long)sysid << kHashSysShift) | (unsigned long long)lin;
    return hash_find(a.hkey, a.hmask, a.table, key, a.err);
}

// The reference's exact FP64 inclusion test (neighbour_visit.hh:88-109).
__device__ __forceinline__ bool exact_inside(const SysDev &S, const TraverseArgs &a,
                                             const double4 &pi, const double4 &pj,
                                             const double *off, float ti_bits,
                                             float tj_bits) {
    const double dx = dadd(dsub(pj.x, pi.x), off[0]);
    const double dy = dadd(dsub(pj.y, pi.y), off[1]);
    const double dz = dadd(dsub(pj.z, pi.z), off[2]);
    const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
    if (!(r2 < S.cutoff_sq)) return false;
    if (S.cutoff_kind == kCutPerAtom) {
        const double cc = dadd(pi.w, pj.w);
        return r2 < dmul(cc, cc);
    }
    if (S.cutoff_kind == kCutPerType) {
        const int ti = __float_as_int(ti_bits), tj = __float_as_int(tj_bits);
        if (ti >= 0 && ti < S.ncutoffs && tj >= 0 && tj < S.ncutoffs)
            return r2 < a.pt64[S.pt_base + ti * S.ncutoffs + tj];
    }
    return true;
}

template <bool FP32>
__device__ __forceinline__ void pair_threshold(const SysDev &S, const TraverseArgs &a,
                                               const Thresh &th, float wi, float wj,
                                               float &lo, float &hi) {
    lo = th.lo_rc;
    hi = th.hi_rc;
    if (S.cutoff_kind == kCutPerAtom) {
        const float cc = wi + wj;
        const float t = cc * cc;
        lo = fminf(lo, t - th.band);
        hi = fminf(hi, t + th.band);
    } else if (S.cutoff_kind == kCutPerType) {
        const int ti = __float_as_int(wi), tj = __float_as_int(wj);
        if (ti >= 0 && ti < S.ncutoffs && tj >= 0 && tj < S.ncutoffs) {
            const float t = a.pt32[S.pt_base + ti * S.ncutoffs + tj];
            lo = fminf(lo, t - th.band);
            hi = fminf(hi, t + th.band);
        }
    }
}

// Emit up to 32 queued pairs (lane L takes entry L).
template <bool FP32>
__device__ __forceinline__ void emit_queue(TravSmem<FP32> &sm, const TraverseArgs &a,
                                           const SysDev &S, int warp, int lane,
                                           int count) {
    if (lane < count) {
        const int32_t e = sm.q[warp][lane];
        const long long slot = sm.qw[warp][lane];
        const int k = e & 0xffff, il = e >> 16;
        const int32_t sj = sm.cand_sj[k];
        const int seg = sm.cand_seg[k];
        const double4 pj = a.pos64[sj];
        const double4 pi = sm.i64[il];
        const int4 aj = a.aux[sj];
        const int4 ai = sm.iaux[il];
        const double dx = dadd(dsub(pj.x, pi.x), sm.seg_off[seg][0]);
        const double dy = dadd(dsub(pj.y, pi.y), sm.seg_off[seg][1]);
        const double dz = dadd(dsub(pj.z, pi.z), sm.seg_off[seg][2]);
        if (a.mat_k > 0) {
            const long long sl = slot - sm.istart[il];
            if (sl < a.mat_k) {
                const long long m = (long long)ai.x * a.mat_k + sl;
                a.mat_idx[m] = (int32_t)(aj.x - S.atom_base);
                a.mat_dist[3 * m + 0] = dx;
                a.mat_dist[3 * m + 1] = dy;
                a.mat_dist[3 * m + 2] = dz;
            }
        } else if (slot < a.capacity) {
            const int32_t il_out = (int32_t)(ai.x - S.atom_base);
            const int32_t jl_out = (int32_t)(aj.x - S.atom_base);
            if (a.first) a.first[slot] = il_out;
            if (a.second) a.second[slot] = jl_out;
            if (a.distvec) {
                a.distvec[3 * slot + 0] = dx;
                a.distvec[3 * slot + 1] = dy;
                a.distvec[3 * slot + 2] = dz;
            }
            if (a.absdist) {
                const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
                a.absdist[slot] = __dsqrt_rn(r2);
            }
            if (a.shift) {
                a.shift[3 * slot + 0] = ai.y - (S.pbc[0] ? aj.y : 0) + sm.seg_m[seg][0];
                a.shift[3 * slot + 1] = ai.z - (S.pbc[1] ? aj.z : 0) + sm.seg_m[seg][1];
                a.shift[3 * slot + 2] = ai.w - (S.pbc[2] ? aj.w : 0) + sm.seg_m[seg][2];
            }
        } else {
            atomicOr(a.err, kErrCapacity);
        }
    }
}

}  // namespace

template <int MODE, bool FP32>
__global__ void __launch_bounds__(kThreads)
k_traverse(TraverseArgs a) {
    constexpr int kCand = TileCfg<FP32>::kCand;
    __shared__ TravSmem<FP32> sm;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned full = 0xffffffffu;
    const int nhome = *a.n_home;

    for (int h = blockIdx.x; h < nhome; h += gridDim.x) {
        const HomeCell hc = a.home[h];
        // System descriptor -> shared memory (broadcast reads in the sweep).
        {
            const int *src = reinterpret_cast<const int *>(a.sys + hc.sys);
            int *dst = reinterpret_cast<int *>(&sm.sys);
            for (int w = tid; w < (int)(sizeof(SysDev) / sizeof(int)); w += kThreads)
                dst[w] = src[w];
        }
        __syncthreads();
        const SysDev &S = sm.sys;
        const int2 hs = a.table[hc.tidx];
        Thresh th;
        if (FP32) {
            const double R = S.cutoff;
            const double M = 2.0 * (double)a.amax[hc.sys] + S.off_max;
            const double band = guard_band(M, R);
            th.lo_rc = __double2float_rd(S.cutoff_sq - band);
            th.hi_rc = __double2float_ru(S.cutoff_sq + band);
            th.band = __double2float_ru(band);
        }
        const int nx = S.nscan[0], ny = S.nscan[1], nz = S.nscan[2];
        const int wx = 2 * nx + 1, wy = 2 * ny + 1;

        for (int ib = hs.x; ib < hs.y; ib += kITile) {
            const int ni = min(kITile, hs.y - ib);
            if (tid < ni) {
                const int si = ib + tid;
                sm.i64[tid] = a.pos64[si];
                sm.i32[tid] = a.pos32[si];
                const int4 ax = a.aux[si];
                sm.iaux[tid] = ax;
                sm.istate[tid] = (MODE == kModeCount) ? 0ll : (long long)a.offsets[ax.x];
                if (MODE == kModeFill) sm.istart[tid] = sm.istate[tid];
            }
            __syncthreads();

            for (int vb = 0; vb < S.nvisit; vb += kSegBatch) {
                const int nseg = min(kSegBatch, S.nvisit - vb);
                // --- segment set-up: one thread per visited offset -----------
                int len = 0;
                if (tid < nseg) {
                    const int v = vb + tid;
                    const int xr = v % wx, rest = v / wx;
                    const int yr = rest % wy, zr = rest / wy;
                    const int off3[3] = {xr - nx, yr - ny, zr - nz};
                    int32_t cj[3], m[3];
                    bool ok = true;
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        int32_t x = hc.c[k] + off3[k];
                        m[k] = 0;
                        if (S.pbc[k]) {
                            m[k] = floor_div(x, S.n[k]);
                            x -= m[k] * S.n[k];
                        } else if (x < 0 || x >= S.n[k]) {
                            ok = false;
                        }
                        cj[k] = x;
                    }
                    int2 sl = make_int2(0, 0);
                    if (ok) sl = cell_lookup(a, S, hc.sys, cj[0], cj[1], cj[2]);
                    len = sl.y - sl.x;
                    sm.seg_b[tid] = sl.x;
                    // neighbour_visit.hh:67,73,80: off3 = z b3; off2 = off3 + y b2;
                    // off = off2 + x b1
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        double o = dmul((double)off3[2], S.bin[2][k]);
                        o = dadd(o, dmul((double)off3[1], S.bin[1][k]));
                        o = dadd(o, dmul((double)off3[0], S.bin[0][k]));
                        sm.seg_off[tid][k] = o;
                        sm.seg_m[tid][k] = m[k];
                    }
                    sm.seg_zero[tid] = (off3[0] == 0 && off3[1] == 0 && off3[2] == 0);
                }
                // block-wide exclusive scan of the segment lengths
                {
                    int incl = len;
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) {
                        int o = __shfl_up_sync(full, incl, d);
                        if (lane >= d) incl += o;
                    }
                    if (lane == 31) sm.scan_warp[warp] = incl;
                    __syncthreads();
                    int wbase = 0, tot = 0;
#pragma unroll
                    for (int w = 0; w < kWarps; w++) {
                        const int ws = sm.scan_warp[w];
                        if (w < warp) wbase += ws;
                        tot += ws;
                    }
                    if (tid < nseg) sm.seg_pref[tid] = wbase + incl - len;
                    if (tid == 0) sm.seg_pref[nseg] = tot;
                    __syncthreads();
                }
                const int total = sm.seg_pref[nseg];

                for (int kb = 0; kb < total; kb += kCand) {
                    const int nk = min(kCand, total - kb);
                    // --- stage candidates ------------------------------------
                    for (int k = tid; k < nk; k += kThreads) {
                        const int kk = kb + k;
                        int lo = 0, hi = nseg - 1;  // last seg with pref <= kk
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if (sm.seg_pref[mid] <= kk)
                                lo = mid;
                            else
                                hi = mid - 1;
                        }
                        const int sj = sm.seg_b[lo] + (kk - sm.seg_pref[lo]);
                        if (FP32) {
                            const float4 p = a.pos32[sj];
                            float4 cv;
                            cv.x = p.x + __double2float_rn(sm.seg_off[lo][0]);
                            cv.y = p.y + __double2float_rn(sm.seg_off[lo][1]);
                            cv.z = p.z + __double2float_rn(sm.seg_off[lo][2]);
                            cv.w = p.w;
                            reinterpret_cast<float4 *>(sm.cand)[k] = cv;
                        } else {
                            reinterpret_cast<double4 *>(sm.cand)[k] = a.pos64[sj];
                        }
                        sm.cand_sj[k] = sj;
                        sm.cand_seg[k] = (uint8_t)lo;
                    }
                    __syncthreads();

                    // --- sweep: warp per atom i ------------------------------
                    int qn = 0;  // warp-uniform queue length (FILL)
                    for (int il = warp; il < ni; il += kWarps) {
                        const int si = ib + il;
                        const float4 pi32 = sm.i32[il];
                        const double4 pi64 = sm.i64[il];
                        long long state = sm.istate[il];
                        for (int k0 = 0; k0 < nk; k0 += 32) {
                            const int k = k0 + lane;
                            bool hit = false;
                            if (k < nk) {
                                const int seg = sm.cand_seg[k];
                                const bool self =
                                    (sm.cand_sj[k] == si) && sm.seg_zero[seg];
                                if (!self) {
                                    if (FP32) {
                                        const float4 cv = reinterpret_cast<const float4 *>(sm.cand)[k];
                                        const float dx = cv.x - pi32.x;
                                        const float dy = cv.y - pi32.y;
                                        const float dz = cv.z - pi32.z;
                                        const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                                        float lo, hi;
                                        pair_threshold<FP32>(S, a, th, pi32.w, cv.w, lo, hi);
                                        if (r2 < lo) {
                                            hit = true;
                                        } else if (r2 < hi) {
                                            const double4 pj = a.pos64[sm.cand_sj[k]];
                                            const float wj = a.pos32[sm.cand_sj[k]].w;
                                            hit = exact_inside(S, a, pi64, pj, sm.seg_off[seg],
                                                               pi32.w, wj);
                                        }
                                    } else {
                                        const double4 pj = reinterpret_cast<const double4 *>(sm.cand)[k];
                                        float wj = 0.f;
                                        if (S.cutoff_kind == kCutPerType)
                                            wj = a.pos32[sm.cand_sj[k]].w;
                                        hit = exact_inside(S, a, pi64, pj, sm.seg_off[seg],
                                                           pi32.w, wj);
                                    }
                                }
                            }
                            const unsigned mask = __ballot_sync(full, hit);
                            if (MODE == kModeCount) {
                                state += __popc(mask);
                            } else if (mask) {
                                const int before = __popc(mask & lanemask_lt());
                                if (hit) {
                                    sm.q[warp][qn + before] = k | (il << 16);
                                    sm.qw[warp][qn + before] = state + before;
                                }
                                state += __popc(mask);
                                qn += __popc(mask);
                                __syncwarp();
                                if (qn >= 32) {
                                    emit_queue<FP32>(sm, a, S, warp, lane, 32);
                                    __syncwarp();
                                    const int rem = qn - 32;
                                    int32_t e = 0;
                                    long long w = 0;
                                    if (lane < rem) {
                                        e = sm.q[warp][32 + lane];
                                        w = sm.qw[warp][32 + lane];
                                    }
                                    __syncwarp();
                                    if (lane < rem) {
                                        sm.q[warp][lane] = e;
                                        sm.qw[warp][lane] = w;
                                    }
                                    __syncwarp();
                                    qn = rem;
                                }
                            }
                        }
                        if (lane == 0) sm.istate[il] = state;
                    }
                    if (MODE == kModeFill && qn > 0) {
                        emit_queue<FP32>(sm, a, S, warp, lane, qn);
                    }
                    __syncthreads();
                }
            }
            // --- per-atom results of this i-tile ---------------------------------
            if (tid < ni) {
                const int4 ax = sm.iaux[tid];
                if (MODE == kModeCount) {
                    a.counts[ax.x] = (int32_t)sm.istate[tid];
                } else {
                    const long long end = (long long)a.offsets[ax.x + 1];
                    if (sm.istate[tid] != end) atomicOr(a.err, kErrInternal);
                    if (a.mat_k > 0) {
                        const long long deg = end - sm.istart[tid];
                        a.mat_count[ax.x] = (int32_t)deg;
                        if (deg > a.mat_k) atomicOr(a.mat_overflow, 1);
                    }
                }
            }
            __syncthreads();
        }
        __syncthreads();
    }
}

template __global__ void k_traverse<kModeCount, true>(TraverseArgs);
template __global__ void k_traverse<kModeCount, false>(TraverseArgs);
template __global__ void k_traverse<kModeFill, true>(TraverseArgs);
template __global__ void k_traverse<kModeFill, false>(TraverseArgs);

cudaError_t launch_bin(const BinArgs &a, cudaStream_t st) {
    if (a.natoms <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((a.natoms + 255) / 256);
    k_bin<<<grid, 256, 0, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_gather(const GatherArgs &a, cudaStream_t st) {
    if (a.natoms <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((a.natoms + 255) / 256);
    k_gather<<<grid, 256, 0, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_traverse(int mode, bool fp32, const TraverseArgs &a, int grid,
                            cudaStream_t st) {
    if (grid <= 0) return cudaSuccess;
    if (mode == kModeCount) {
        if (fp32)
            k_traverse<kModeCount, true><<<grid, kThreads, 0, st>>>(a);
        else
            k_traverse<kModeCount, false><<<grid, kThreads, 0, st>>>(a);
    } else {
        if (fp32)
            k_traverse<kModeFill, true><<<grid, kThreads, 0, st>>>(a);
        else
            k_traverse<kModeFill, false><<<grid, kThreads, 0, st>>>(a);
    }
    count_launch();
    return cudaGetLastError();
}

}  // namespace nbl
