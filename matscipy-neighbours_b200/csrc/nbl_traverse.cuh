// nbl_traverse.cuh -- the pair passes k_count and k_fill, as templates over
// the launch shape (warps per CTA, candidates staged per warp, atoms swept
// per pass).  Included by the translation units that instantiate and launch
// them (nbl_trav_*.cu); everything here has internal linkage, so each unit
// carries only the instantiations it launches.
//
// Shared memory is dynamic: a CTA holds one per-warp state block per warp
// (plus, for the force sink, the warps' per-atom sums), sized by
// count_smem_bytes / fill_smem_bytes below.
#pragma once

#include <climits>
#include <cstdint>
#include <mutex>
#include <set>
#include <type_traits>
#include <utility>

#include <cuda_runtime.h>

#include "nbl_build.cuh"
#include "nbl_internal.cuh"

namespace nbl {
namespace {

// ---------------------------------------------------------------------------
// The pair passes: k_count and k_fill
// ---------------------------------------------------------------------------
//
// Both take one work item (home cell x i-tile of up to 32 atoms; the tile
// size is a launch parameter) per WARP (each warp claims its next item with
// an atomic ticket, issued while the current item runs, or takes items at a
// fixed warp stride; a CTA is 2, 4 or 8 independent warps, so there is no
// block-wide barrier).  Per item, one lane per visited neighbour offset
// reads the offset vector (FP64, reference order, from the per-system visit
// table), the wrap counts and the cell slice, and a warp scan turns slice
// lengths into candidate positions (the "segment batch").
//
// A run (WorkItem::run > 1, the RUN instantiations) is an item of several
// home cells along x: its segments are the run's rows of neighbour cells,
// each atom keeps only the segments within one cell of its own (its own
// 3 x 3 x 3 block, in order), and D is formed with the offset of the atom's
// own cell offset, so every row is exactly the one-cell item's row.
//
// k_count stages the candidates in shared memory as FP32 positions in the
// home-cell frame (lane = segment: each copies its cell's run of sorted
// atoms) and sweeps them against the tile's atoms, GROUP atoms per pass
// (independent FMA chains), 32 candidates per __ballot_sync.  Each chunk's
// hit mask is popc'ed into the atom's count and, when the item fits the mask
// pool, stored as one 32-bit word per (atom, chunk).
//
// k_fill turns hit words back into pairs lane-parallel: for a window of atoms
// it builds the prefix of the words' popcounts and keeps the atoms whose pairs
// fit kPosTab; each word then writes its set bits' (candidate, atom) codes at
// their output positions (lane = word, ffs), so lane L of each round finds
// pair P = P0 + L with one shared-memory load (a single atom with more pairs
// searches: binary search over the prefix, then an n-th-set-bit search).  The pair (exact FP64
// D, d and S) goes to row_start + rank, so consecutive lanes write
// consecutive slots; the next round's j-side loads are issued before this
// round's stores.  Items without pool words (pool full, more than
// kMaskBatches segment batches) recompute the words with the count's sweep
// first.
namespace {

constexpr int kSeg = 32;         // visited offsets per batch (one per lane)
constexpr int kITile = 32;       // atoms i per i-tile
constexpr int kWinWords = 256;   // hit words per emission window
constexpr int kRange = kWinWords * 32;  // candidates per emission range
constexpr float kFarCand = 1.0e18f;     // padding candidate
constexpr float kFarAtom = -1.0e18f;    // padding atom (never near a padding candidate)

// Resident CTAs per SM each pair pass is compiled for (the register budget):
// 24 count warps and 20 fill warps per SM (16 with 8-warp fill CTAs).
constexpr int count_min_blocks(int warps) { return 24 / warps; }
constexpr int fill_min_blocks(int warps) { return warps == 2 ? 10 : (warps == 4 ? 5 : 2); }

template <bool FP32>
using CandT = typename std::conditional<FP32, float4, double4>::type;

template <bool FP32>
struct FillTile {
    static constexpr int kCand = FP32 ? 64 : 32;
};

// One visited segment, read by the fill with three wide loads: its offset
// vector (FP64, the reference's order), the image shift of the visited cell
// and bj = (first sorted atom of the cell) - (first candidate index of the
// segment), so candidate kk of the segment is sorted atom bj + kk.
struct __align__(16) SegRec {
    double off[3];
    int32_t m[3];
    int32_t bj;
};

struct SegSmem {
    SegRec rec[kSeg];
    float off32[kSeg][3];
    int32_t b[kSeg];
    int32_t pref[kSeg + 1];
    int8_t xo[kSeg];    // runs: the segment's x cell offset from the run's first cell
    uint8_t row[kSeg];  // runs: its (z, y) offset row, (dz + 1) * 3 + dy + 1
};

// A segment record's values (offset vector and image shift) in registers.
struct SegVals {
    double o0, o1, o2;
    int32_t m0, m1, m2;
};
__device__ __forceinline__ SegVals seg_vals(const SegRec &g) {
    const double2 o01 = *reinterpret_cast<const double2 *>(&g.off[0]);
    const int4 o2m = *reinterpret_cast<const int4 *>(&g.off[2]);
    SegVals v;
    v.o0 = o01.x;
    v.o1 = o01.y;
    v.o2 = __hiloint2double(o2m.y, o2m.x);
    v.m0 = o2m.z;
    v.m1 = o2m.w;
    v.m2 = g.m[2];
    return v;
}

template <bool FP32, int CAND>
struct __align__(16) CountSmem {
    SegSmem sg;
    CandT<FP32> cand[CAND];
    float4 i32[kITile];
    int32_t iatom[kITile];
    int32_t isi[kITile];       // sorted index of each (in-range) atom of the tile
    int32_t icount[kITile];
    int8_t ht[kITile];         // runs: each atom's home cell within the run
};
static_assert(6 * (4 * sizeof(CountSmem<true, 384>) + 1024) <= 233472,
              "six 4-warp count CTAs per SM fit the SM's shared memory");

constexpr int kCandTab = 1024;   // candidates with a segment-table entry (fill)
constexpr int kPosTab = 640;     // pairs per window with a position table (fill)
static_assert(kRange <= 8192 && kITile <= 32,
              "position-table entries hold the candidate in 13 bits, the atom in 5");

// Per-warp fill state, about 9.6 KB, so that five 4-warp CTAs fit an SM
// (the force sink's sums live in a separate array of the force-sink kernel).
template <bool FP32>
struct __align__(16) FillSmem {
    SegSmem sg;
    double4 i64[kITile];
    int4 iaux[kITile];
    int32_t isi[kITile];       // sorted index of each (in-range) atom of the tile
    long long icur[kITile];
    long long abase[kITile];   // output slot of window position 0 of each window atom
    uint32_t mw[kWinWords];
    int32_t mpre[kWinWords + 1];
    union {
        uint32_t ptab[kPosTab];  // window position -> candidate | atom << 13 (small windows)
        CandT<FP32> cand[FillTile<FP32>::kCand];  // staged candidates (recomputed words)
    };
    uint8_t cand_seg[kCandTab];     // segment of each of the batch's first candidates
    int8_t ht[kITile];              // runs: each atom's home cell within the run
};
static_assert(5 * (4 * sizeof(FillSmem<true>) + 4 * 32 * 32 + 1024) <= 233472 &&
                  5 * (4 * sizeof(FillSmem<false>) + 4 * 32 * 32 + 1024) <= 233472,
              "five 4-warp fill CTAs per SM (force-sink sums included) fit the SM's "
              "shared memory");

// Per-home-cell constants kept in registers.
struct Hot {
    float lo_rc, hi_rc, band;
    double cutoff_sq;
    int pbc_bits;
    int ncut;
    int pt_base;
    int vrun;  // runs: the system's first visit-table entry; -1: a single cell
    int64_t atom_base;
};

struct Home {
    int32_t cc[3];  // folded coordinates of the (first) home cell
    int sys;
    const SysDev *S;
    Hot H;
    int nvisit;
    int run;        // home cells of the item
};

// RUN: the kernel instantiation that takes runs (items of several home
// cells); without it every item is one cell and the run code folds away.
template <bool FP32, bool RUN>
__device__ __forceinline__ Home load_home(const TraverseArgs &a, const WorkItem &w) {
    Home c;
    const int run = RUN ? w.run : 1;
    c.cc[0] = w.c[0];
    c.cc[1] = w.c[1];
    c.cc[2] = w.c[2];
    c.sys = w.sys;
    c.S = a.sys + w.sys;
    const SysDev &S = *c.S;
    c.H.vrun = run > 1 ? (int)S.visit_base : -1;
    c.H.lo_rc = c.H.hi_rc = c.H.band = 0.f;
    if (FP32) {
        const double R = S.cutoff;
        double M = 2.0 * (double)a.amax[w.sys] + S.off_max;
        if (run > 1) {
            // a run stages candidates and atoms in its first cell's frame:
            // candidate offsets reach (run - 1) more cells along x, atom
            // offsets up to run - 1 cells
            const double bx = fmax(fabs(S.bin[0][0]), fmax(fabs(S.bin[0][1]), fabs(S.bin[0][2])));
            M = dadd(M, dmul(2.0 * (double)(run - 1), bx) * (1.0 + 1e-12));
        }
        const double band = guard_band(M, R);
        c.H.lo_rc = __double2float_rd(S.cutoff_sq - band);
        c.H.hi_rc = __double2float_ru(S.cutoff_sq + band);
        c.H.band = __double2float_ru(band);
    }
    c.H.cutoff_sq = S.cutoff_sq;
    c.H.pbc_bits = (S.pbc[0] ? 1 : 0) | (S.pbc[1] ? 2 : 0) | (S.pbc[2] ? 4 : 0);
    c.H.ncut = S.ncutoffs;
    c.H.pt_base = S.pt_base;
    c.H.atom_base = S.atom_base;
    c.run = run;
    c.nvisit = run > 1 ? 9 * (run + 2) : S.nvisit;
    return c;
}

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

// Segment batch vb of a home cell: one lane per visited offset
// (neighbour_visit.hh:63-84).  Returns the batch size, its candidate total
// and the index of the zero-offset segment (-1 if not in this batch).
__device__ __forceinline__ void setup_segments(SegSmem &sg, const TraverseArgs &a,
                                               const Home &c, int vb, int lane, int &nseg,
                                               int &total, int &zs) {
    const unsigned full = 0xffffffffu;
    const SysDev &S = *c.S;
    const int nx = S.nscan[0], ny = S.nscan[1], nz = S.nscan[2];
    const int wx = 2 * nx + 1, wy = 2 * ny + 1;
    nseg = min(kSeg, c.nvisit - vb);
    int len = 0;
    bool zero = false;
    if (lane < nseg) {
        const int v = vb + lane;
        int off3[3];
        double offd[3];
        float off32[3];
        uint8_t vrow = 0;
        if (c.run > 1) {
            // a run: rows (dz, dy) in the reference's order, each the run's
            // cells plus one on either side, x ascending (so each atom sees its
            // own 3 x 3 x 3 block in z/y/x order)
            const int wr = c.run + 2;
            const int xr = v % wr, rest = v / wr;
            off3[0] = xr - 1;
            off3[1] = rest % 3 - 1;
            off3[2] = rest / 3 - 1;
            vrow = (uint8_t)rest;
            visit_offset(S, off3, offd);
#pragma unroll
            for (int k = 0; k < 3; k++) off32[k] = __double2float_rn(offd[k]);
        } else if (S.visit_base >= 0) {
            const VisitDev &e = a.visit[S.visit_base + v];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                off3[k] = e.d[k];
                offd[k] = e.off[k];
                off32[k] = e.off32[k];
            }
        } else {
            const int xr = v % wx, rest = v / wx;
            const int yr = rest % wy, zr = rest / wy;
            off3[0] = xr - nx;
            off3[1] = yr - ny;
            off3[2] = zr - nz;
            visit_offset(S, off3, offd);
#pragma unroll
            for (int k = 0; k < 3; k++) off32[k] = __double2float_rn(offd[k]);
        }
        int32_t cj[3], m[3];
        bool ok = true;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            int32_t x = c.cc[k] + off3[k];
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
                ok = false;
            }
            cj[k] = x;
        }
        int2 sl = make_int2(0, 0);
        if (ok) sl = cell_lookup(a, S, c.sys, cj[0], cj[1], cj[2]);
        if (checked_fail(sl.x < 0 || sl.y < sl.x || (long long)sl.y > a.natoms, a.err))
            sl = make_int2(0, 0);
        len = sl.y - sl.x;
        sg.b[lane] = sl.x;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            sg.rec[lane].off[k] = offd[k];
            sg.off32[lane][k] = off32[k];
            sg.rec[lane].m[k] = m[k];
        }
        if (c.run > 1) {
            sg.xo[lane] = (int8_t)off3[0];
            sg.row[lane] = vrow;
        }
        zero = c.run == 1 && off3[0] == 0 && off3[1] == 0 && off3[2] == 0;
    }
    int incl = len;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int o = __shfl_up_sync(full, incl, d);
        if (lane >= d) incl += o;
    }
    total = __shfl_sync(full, incl, 31);
    if (lane < nseg) {
        sg.pref[lane] = incl - len;
        sg.rec[lane].bj = sg.b[lane] - (incl - len);
    }
    if (lane == 0) sg.pref[nseg] = total;
    const unsigned zm = __ballot_sync(full, zero);
    zs = zm ? __ffs(zm) - 1 : -1;
    __syncwarp();
}

// Segment of candidate kk of the current batch.
__device__ __forceinline__ int seg_of(const SegSmem &sg, int nseg, int kk) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (sg.pref[mid] <= kk)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Stage candidates kb .. kb+nk of the batch, padded to nkp with far points.
// Short cell runs (the usual case): lane = segment, each copying its cell's
// run of consecutive sorted atoms.  Long runs: lane = candidate, the lane's
// segment found once by search and then advanced as its candidate grows.
template <bool FP32>
__device__ __forceinline__ void stage_segs(CandT<FP32> *cand, const SegSmem &sg,
                                           const TraverseArgs &a, int nseg, int kb, int nk,
                                           int nkp, int lane) {
    __syncwarp();
    if (sg.pref[nseg] > 48 * nseg) {
        int seg = lane < nk ? seg_of(sg, nseg, kb + lane) : 0;
        for (int k = lane; k < nk; k += 32) {
            const int kk = kb + k;
            while (seg + 1 < nseg && sg.pref[seg + 1] <= kk) seg++;
            const int sj = sg.b[seg] + (kk - sg.pref[seg]);
            if constexpr (FP32) {
                const float4 p = a.pos32[sj];
                cand[k] = make_float4(p.x + sg.off32[seg][0], p.y + sg.off32[seg][1],
                                      p.z + sg.off32[seg][2], p.w);
            } else {
                cand[k] = a.pos64[sj];
            }
        }
    } else if (lane < nseg) {
        const int s0 = max(sg.pref[lane], kb), s1 = min(sg.pref[lane + 1], kb + nk);
        const int jb = sg.b[lane] - sg.pref[lane];
        if constexpr (FP32) {
            const float ox = sg.off32[lane][0], oy = sg.off32[lane][1], oz = sg.off32[lane][2];
#pragma unroll 4
            for (int kk = s0; kk < s1; kk++) {
                const float4 p = a.pos32[jb + kk];
                cand[kk - kb] = make_float4(p.x + ox, p.y + oy, p.z + oz, p.w);
            }
        } else {
#pragma unroll 4
            for (int kk = s0; kk < s1; kk++) cand[kk - kb] = a.pos64[jb + kk];
        }
    }
    for (int k = nk + lane; k < nkp; k += 32) {
        if constexpr (FP32)
            cand[k] = make_float4(kFarCand, kFarCand, kFarCand, 0.f);
        else
            cand[k] = make_double4(kFarCand, kFarCand, kFarCand, 0.0);
    }
    __syncwarp();
}

// FP32 staging for the count, as stage_segs but without a dependent global
// load per candidate: with short cell runs each lane (segment) starts
// asynchronous copies of its whole run, waits for them, and adds its
// segment's offset to the run in shared memory.
__device__ __forceinline__ void stage_segs_async(float4 *cand, const SegSmem &sg,
                                                 const TraverseArgs &a, int nseg, int kb, int nk,
                                                 int nkp, int lane) {
    if (sg.pref[nseg] > 48 * nseg) {
        stage_segs<true>(cand, sg, a, nseg, kb, nk, nkp, lane);
        return;
    }
    __syncwarp();
    if (lane < nseg) {
        const int s0 = max(sg.pref[lane], kb), s1 = min(sg.pref[lane + 1], kb + nk);
        const int jb = sg.b[lane] - sg.pref[lane];
        for (int kk = s0; kk < s1; kk++) cp_async16(&cand[kk - kb], &a.pos32[jb + kk]);
        cp_async_wait();
        const float ox = sg.off32[lane][0], oy = sg.off32[lane][1], oz = sg.off32[lane][2];
#pragma unroll 4
        for (int kk = s0; kk < s1; kk++) {
            const float4 p = cand[kk - kb];
            cand[kk - kb] = make_float4(p.x + ox, p.y + oy, p.z + oz, p.w);
        }
    }
    for (int k = nk + lane; k < nkp; k += 32)
        cand[k] = make_float4(kFarCand, kFarCand, kFarCand, 0.f);
    __syncwarp();
}

// The reference's exact FP64 inclusion test (neighbour_visit.hh:88-109).
template <int KIND>
__device__ __forceinline__ bool exact_inside(const Hot &H, const TraverseArgs &a,
                                             const double4 &pi, const double4 &pj,
                                             const double *off, float ti_bits,
                                             float tj_bits) {
    const double dx = dadd(dsub(pj.x, pi.x), off[0]);
    const double dy = dadd(dsub(pj.y, pi.y), off[1]);
    const double dz = dadd(dsub(pj.z, pi.z), off[2]);
    const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
    if (!(r2 < H.cutoff_sq)) return false;
    if (KIND == kCutPerAtom) {
        const double cc = dadd(pi.w, pj.w);
        return r2 < dmul(cc, cc);
    }
    if (KIND == kCutPerType) {
        const int ti = __float_as_int(ti_bits), tj = __float_as_int(tj_bits);
        if (ti >= 0 && ti < H.ncut && tj >= 0 && tj < H.ncut)
            return r2 < a.pt64[H.pt_base + ti * H.ncut + tj];
    }
    return true;
}

// Guard-band candidate kk of the batch for atom si, decided in FP64 (cold).
// In a run (H.vrun >= 0) the atom (home cell t of the run) only has the
// segments within one cell of its own along x, with the offset vector of its
// own cell offset (the reference's visit of that home cell).
template <int KIND, bool RUN>
__device__ __noinline__ bool resolve_exact(const SegSmem &sg, const TraverseArgs &a,
                                           const Hot &H, const SysDev *S, int nseg, int kk,
                                           int si, float wi, int t) {
    const int seg = seg_of(sg, nseg, kk);
    const int32_t sj = sg.b[seg] + (kk - sg.pref[seg]);
    if (RUN && H.vrun >= 0) {
        const int dx = (int)sg.xo[seg] - t;
        if (dx < -1 || dx > 1) return false;
        const int d[3] = {dx, (int)sg.row[seg] % 3 - 1, (int)sg.row[seg] / 3 - 1};
        double off[3];
        visit_offset(*S, d, off);
        return exact_inside<KIND>(H, a, a.pos64[si], a.pos64[sj], off, wi, a.pos32[sj].w);
    }
    return exact_inside<KIND>(H, a, a.pos64[si], a.pos64[sj], sg.rec[seg].off, wi,
                              a.pos32[sj].w);
}

// Runs: the home cell (0 .. run - 1) of sorted atom si, found among the run's
// cell slices (every lane takes part; lane t < run reads cell t's slice).
__device__ __forceinline__ int run_home_of(const TraverseArgs &a, const WorkItem &w, int si,
                                           int lane) {
    int2 sl = make_int2(0, 0);
    if (lane < w.run) sl = a.table[w.tidx + lane];
    int t = 0;
    for (int u = 0; u < w.run; u++) {
        const int b = __shfl_sync(0xffffffffu, sl.x, u);
        const int e = __shfl_sync(0xffffffffu, sl.y, u);
        if (si >= b && si < e) t = u;
    }
    return t;
}

// Runs: (first candidate index - first sorted atom) of home cell t's own
// segment (zero offset) if it is in the batch starting at segment vb, else
// INT_MIN / 2 (so that kself + si stays negative).
__device__ __forceinline__ int run_self_base(const SegSmem &sg, int run, int vb, int nseg,
                                             int t) {
    const int zv = 4 * (run + 2) + t + 1 - vb;  // row (0, 0), x offset t
    return (zv >= 0 && zv < nseg) ? sg.pref[zv] - sg.b[zv] : INT_MIN / 2;
}

// Runs: FP32 offset of home cell t from the run's first cell (the frame the
// run's candidates and atoms are staged in).
__device__ __forceinline__ float3 run_frame32(const SysDev &S, int t) {
    const int d[3] = {t, 0, 0};
    double o[3];
    visit_offset(S, d, o);
    return make_float3(__double2float_rn(o[0]), __double2float_rn(o[1]),
                       __double2float_rn(o[2]));
}

// FP32 thresholds for one (atom, candidate) pair.
template <int KIND>
__device__ __forceinline__ void thresholds(const Hot &H, const TraverseArgs &a, float wi,
                                           float wj, float &lo, float &hi) {
    lo = H.lo_rc;
    hi = H.hi_rc;
    if (KIND == kCutPerAtom) {
        const float cc = wi + wj;
        const float t = cc * cc;
        lo = fminf(lo, t - H.band);
        hi = fminf(hi, t + H.band);
    } else if (KIND == kCutPerType) {
        const int ti = __float_as_int(wi), tj = __float_as_int(wj);
        if (ti >= 0 && ti < H.ncut && tj >= 0 && tj < H.ncut) {
            const float t = a.pt32[H.pt_base + ti * H.ncut + tj];
            lo = fminf(lo, t - H.band);
            hi = fminf(hi, t + H.band);
        }
    }
}

// Hit mask of one staged 32-candidate chunk (tile positions k0..k0+31) for one
// atom: FP32 filter + FP64 guard band, or plain FP64.
template <bool FP32, int KIND, bool RUN>
__device__ __forceinline__ unsigned chunk_mask(const CandT<FP32> *cand, const SegSmem &sg,
                                               const TraverseArgs &a, const Hot &H,
                                               const SysDev *S, int nseg, int kb, int k0,
                                               int lane, int kself_tile, int si,
                                               const float4 &pi32, const double4 &pi64,
                                               int t) {
    const unsigned full = 0xffffffffu;
    const int k = k0 + lane;
    const bool notself = k != kself_tile;
    if constexpr (FP32) {
        const float4 cv = cand[k];
        const float dx = cv.x - pi32.x;
        const float dy = cv.y - pi32.y;
        const float dz = cv.z - pi32.z;
        const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
        float lo, hi;
        thresholds<KIND>(H, a, pi32.w, cv.w, lo, hi);
        unsigned mask = __ballot_sync(full, (r2 < lo) && notself);
        const bool amb = !(r2 < lo) && (r2 < hi) && notself;
        if (__any_sync(full, amb)) {
            bool h2 = false;
            if (amb) h2 = resolve_exact<KIND, RUN>(sg, a, H, S, nseg, kb + k, si, pi32.w, t);
            mask |= __ballot_sync(full, h2);
        }
        return mask;
    } else {
        bool hit = false;
        const double4 pj = cand[k];
        if (notself && pj.x != (double)kFarCand) {
            const int seg = seg_of(sg, nseg, kb + k);
            float tj = 0.f;
            if (KIND == kCutPerType) tj = a.pos32[sg.b[seg] + (kb + k - sg.pref[seg])].w;
            hit = exact_inside<KIND>(H, a, pi64, pj, sg.rec[seg].off, pi32.w, tj);
        }
        return __ballot_sync(full, hit);
    }
}

// The warp's first work item: a ticket from a.item_next, else the warp index.
__device__ __forceinline__ int first_item(const TraverseArgs &a, int gwarp, int lane) {
    if (a.item_next == nullptr) return gwarp;
    int t = 0;
    if (lane == 0) t = atomicAdd(a.item_next, 1);
    return __shfl_sync(0xffffffffu, t, 0);
}

// A warp's walk over the work items, in ticket order (one atomic per item,
// claimed one item ahead of its use) or at a fixed warp stride.  While the
// current item runs, the record of the next one (and, for the fill, its first
// mask-pool reference) is already on its way:
//     ItemLoop L(...);
//     while (L.it < nitems) { L.prefetch(...); <item L.it, L.rec, L.hm>; L.step(); }
struct ItemLoop {
    int it, nit;
    int tk;                 // lane 0: the ticket after nit
    WorkItem rec, nrec;
    long long hm, nhm;      // first mask reference of it / nit (-1: none)

    __device__ ItemLoop(const TraverseArgs &a, int gwarp, int nitems, int lane, bool want_hm) {
        it = first_item(a, gwarp, lane);
        tk = 0;
        if (a.item_next != nullptr && lane == 0) tk = atomicAdd(a.item_next, 1);
        nit = 0;
        hm = nhm = -1;
        if (it < nitems) {
            rec = a.items[it];
            if (want_hm && a.mask_pool != nullptr)
                hm = a.home_mask[(long long)it * kMaskBatches];
        }
    }
    __device__ void prefetch(const TraverseArgs &a, int nwarps, int nitems, int lane,
                             bool want_hm) {
        if (a.item_next != nullptr) {
            nit = __shfl_sync(0xffffffffu, tk, 0);
            if (lane == 0) tk = atomicAdd(a.item_next, 1);
        } else {
            nit = it + nwarps;
        }
        nhm = -1;
        if (nit < nitems) {
            nrec = a.items[nit];
            if (want_hm && a.mask_pool != nullptr)
                nhm = a.home_mask[(long long)nit * kMaskBatches];
        }
    }
    __device__ void step() {
        it = nit;
        rec = nrec;
        hm = nhm;
    }
};

// Whether every atom produces rows (no nbl_set_atom_range split).
__device__ __forceinline__ bool all_rows_of(const TraverseArgs &a) {
    return a.i_lo <= 0 && a.i_hi >= (1ll << 40);
}

// Checked build: the work item's tile lies inside the sorted atoms.
__device__ __forceinline__ bool item_bad(const TraverseArgs &a, const WorkItem &w) {
    return checked_fail(w.ib < 0 || w.nt < 0 || w.nt > kITile ||
                            (long long)w.ib + w.nt > a.natoms,
                        a.err);
}

// Checked build: hit word `idx` lies inside the pool.
__device__ __forceinline__ bool word_bad(const TraverseArgs &a, long long idx) {
    return checked_fail(idx < 0 || idx >= a.mask_cap, a.err);
}

// Position of the (r+1)-th set bit of w (r < popc(w)).
__device__ __forceinline__ int nth_set_bit(unsigned w, int r) {
    int pos = 0;
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) {
        const unsigned low = w & ((1u << sh) - 1u);
        const int c = __popc(low);
        if (r >= c) {
            r -= c;
            w >>= sh;
            pos += sh;
        } else {
            w = low;
        }
    }
    return pos;
}

// w / n for 0 <= w < 2^20 and small n, without an integer division.
__device__ __forceinline__ int div_small(int w, int n, float inv_n) {
    int q = __float2int_rz((float)w * inv_n);
    if (q * n > w) q--;
    if ((q + 1) * n <= w) q++;
    return q;
}

}  // namespace

// The count pass for one warp of the calling CTA: global warp `gwarp` of
// `nwarps` takes work items (by ticket, else at that stride); `smem_base` is
// the CTA's per-warp count state (one CountSmem per warp of the CTA).
template <bool FP32, int KIND, int GROUP, int CAND, bool RUN>
__device__ __forceinline__ void count_items(const TraverseArgs &a, unsigned char *smem_base,
                                            int gwarp, int nwarps) {
    constexpr int kCand = CAND;
    CountSmem<FP32, CAND> *smem = reinterpret_cast<CountSmem<FP32, CAND> *>(smem_base);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    CountSmem<FP32, CAND> &sm = smem[warp];
    const unsigned full = 0xffffffffu;
    const int nitems = *a.n_items;

    const bool all_rows = all_rows_of(a);
    ItemLoop L(a, gwarp, nitems, lane, false);
    while (L.it < nitems) {
        L.prefetch(a, nwarps, nitems, lane, false);
        const int it = L.it;
        const Home c = load_home<FP32, RUN>(a, L.rec);
        const Hot &H = c.H;
        long long mbase = -1;

        do {
            const int ib = L.rec.ib;
            if (item_bad(a, L.rec)) break;
            // The tile's atoms whose original index lies in [i_lo, i_hi),
            // compacted in order (all of them unless the rows are split); with
            // all rows they are copied asynchronously and land during the
            // segment set-up.  In a run, each atom's home cell and FP32 frame
            // offset (its cell's offset from the run's first cell).
            const int t_l = c.run > 1 ? run_home_of(a, L.rec, ib + lane, lane) : 0;
            int ni;
            if (all_rows) {
                ni = L.rec.nt;
                if (lane < ni) {
                    cp_async16(&sm.i32[lane], &a.pos32[ib + lane]);
                    cp_async4(&sm.iatom[lane], &a.aux[ib + lane].x);
                    sm.isi[lane] = ib + lane;
                    sm.icount[lane] = 0;
                    if (RUN) sm.ht[lane] = (int8_t)t_l;
                }
            } else {
                const int nt = L.rec.nt;
                int ax = 0;
                bool in = false;
                if (lane < nt) {
                    ax = a.aux[ib + lane].x;
                    in = ax >= a.i_lo && ax < a.i_hi;
                }
                const unsigned im = __ballot_sync(full, in);
                ni = __popc(im);
                if (in) {
                    const int c2 = __popc(im & lanemask_lt());
                    float4 p = a.pos32[ib + lane];
                    if (c.run > 1) {
                        const float3 fo = run_frame32(*c.S, t_l);
                        p.x += fo.x;
                        p.y += fo.y;
                        p.z += fo.z;
                    }
                    sm.i32[c2] = p;
                    sm.iatom[c2] = ax;
                    sm.isi[c2] = ib + lane;
                    sm.icount[c2] = 0;
                    sm.ht[c2] = (int8_t)t_l;
                }
                __syncwarp();
            }
            if (ni == 0) break;
            for (int vb = 0; vb < c.nvisit; vb += kSeg) {
                int nseg, total, zs;
                setup_segments(sm.sg, a, c, vb, lane, nseg, total, zs);
                cp_async_wait();
                __syncwarp();
                if (c.run > 1 && all_rows && vb == 0) {  // the copied atoms into the run's frame
                    if (lane < ni) {
                        const float3 fo = run_frame32(*c.S, sm.ht[lane]);
                        float4 p = sm.i32[lane];
                        p.x += fo.x;
                        p.y += fo.y;
                        p.z += fo.z;
                        sm.i32[lane] = p;
                    }
                    __syncwarp();
                }
                const int nchunks_all = (total + 31) >> 5;
                // One word region per (work item, segment batch): (atoms of the
                // i-tile) x (chunks of the batch's candidate list).
                mbase = -1;
                if (a.mask_pool != nullptr && vb / kSeg < kMaskBatches) {
                    long long base = -1;
                    if (lane == 0) {
                        const long long words = (long long)ni * nchunks_all;
                        const unsigned long long b =
                            atomicAdd(a.mask_cursor, (unsigned long long)words);
                        if ((long long)b + words <= a.mask_cap) base = (long long)b;
                    }
                    base = __shfl_sync(full, base, 0);
                    if (lane == 0)
                        a.home_mask[(long long)it * kMaskBatches + vb / kSeg] =
                            base >= 0 ? mask_ref(base, nchunks_all) : -1ll;
                    mbase = base;
                }
                // candidate index of atom si itself at offset 0 is kself0 + si
                const int kself0 = (zs >= 0) ? sm.sg.pref[zs] - sm.sg.b[zs] : INT_MIN / 2;

                for (int kb = 0; kb < total; kb += kCand) {
                    const int nk = min(kCand, total - kb);
                    const int nkp = (nk + 31) & ~31;
                    const int nck = nkp >> 5;
                    if constexpr (FP32)
                        stage_segs_async(sm.cand, sm.sg, a, nseg, kb, nk, nkp, lane);
                    else
                        stage_segs<FP32>(sm.cand, sm.sg, a, nseg, kb, nk, nkp, lane);
                    if constexpr (FP32) {
                        // GROUP atoms per pass over the tile
                        for (int g0 = 0; g0 < ni; g0 += GROUP) {
                            float4 pg[GROUP];
                            int ks[GROUP], cnt[GROUP];
                            unsigned mw[GROUP];
#pragma unroll
                            for (int g = 0; g < GROUP; g++) {
                                const bool v = g0 + g < ni;
                                pg[g] = v ? sm.i32[g0 + g]
                                          : make_float4(kFarAtom, kFarAtom, kFarAtom, 0.f);
                                const int ks0 = c.run == 1
                                                    ? kself0
                                                    : run_self_base(sm.sg, c.run, vb, nseg,
                                                                    v ? sm.ht[g0 + g] : 0);
                                ks[g] = v ? ks0 + sm.isi[g0 + g] - kb : -1;
                                cnt[g] = 0;
                                mw[g] = 0u;
                            }
                            // atoms in pairs for the packed (f32x2) arithmetic:
                            // x - p == x + (-p) exactly, and the packed ops round
                            // each half like the scalar fmaf chain
                            constexpr int kHalf = GROUP / 2;
                            float2 nx[kHalf], ny[kHalf], nz[kHalf];
#pragma unroll
                            for (int h = 0; h < kHalf; h++) {
                                nx[h] = make_float2(-pg[2 * h].x, -pg[2 * h + 1].x);
                                ny[h] = make_float2(-pg[2 * h].y, -pg[2 * h + 1].y);
                                nz[h] = make_float2(-pg[2 * h].z, -pg[2 * h + 1].z);
                            }
                            // blocks of up to 32 chunks: lane L keeps chunk cb + L's hit
                            // word of each atom; the block's counts and its pool words
                            // are taken once at its end
                            for (int cb = 0; cb < nck; cb += 32) {
                                const int ce = min(nck, cb + 32);
#pragma unroll
                                for (int g = 0; g < GROUP; g++) mw[g] = 0u;
                                for (int ch = cb; ch < ce; ch++) {
                                    const int k = ch * 32 + lane;
                                    const float4 cv = sm.cand[k];
                                    unsigned m[GROUP];
                                    bool amb_any = false, amb[GROUP];
                                    float r2g[GROUP];
                                    const float2 cx = make_float2(cv.x, cv.x);
                                    const float2 cy = make_float2(cv.y, cv.y);
                                    const float2 cz = make_float2(cv.z, cv.z);
#pragma unroll
                                    for (int h = 0; h < kHalf; h++) {
                                        const float2 dx = __fadd2_rn(cx, nx[h]);
                                        const float2 dy = __fadd2_rn(cy, ny[h]);
                                        const float2 dz = __fadd2_rn(cz, nz[h]);
                                        const float2 r2 = __ffma2_rn(
                                            dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
                                        r2g[2 * h] = r2.x;
                                        r2g[2 * h + 1] = r2.y;
                                    }
                                    if (KIND != kCutScalar) {
                                        // Pair thresholds never exceed the binning
                                        // cutoff's: a chunk with no candidate inside it
                                        // for any atom of the sweep has no hit and no
                                        // guard-band candidate, so the per-pair
                                        // thresholds are skipped (its words stay 0).
                                        float r2min = r2g[0];
#pragma unroll
                                        for (int g = 1; g < GROUP; g++) r2min = fminf(r2min, r2g[g]);
                                        if (!__any_sync(full, r2min < H.hi_rc)) continue;
                                    }
#pragma unroll
                                    for (int g = 0; g < GROUP; g++) {
                                        const float r2 = r2g[g];
                                        float lo, hi;
                                        thresholds<KIND>(H, a, pg[g].w, cv.w, lo, hi);
                                        m[g] = __ballot_sync(full, r2 < lo);
                                        amb[g] = !(r2 < lo) && (r2 < hi);
                                        amb_any |= amb[g];
                                    }
                                    if (__any_sync(full, amb_any)) {
#pragma unroll
                                        for (int g = 0; g < GROUP; g++) {
                                            bool h2 = false;
                                            if (amb[g])
                                                h2 = resolve_exact<KIND, RUN>(
                                                    sm.sg, a, H, RUN ? c.S : nullptr, nseg,
                                                    kb + k, sm.isi[g0 + g], pg[g].w,
                                                    RUN ? (int)sm.ht[g0 + g] : 0);
                                            m[g] |= __ballot_sync(full, h2);
                                        }
                                    }
                                    const bool mine = lane == ch - cb;
#pragma unroll
                                    for (int g = 0; g < GROUP; g++) mw[g] = mine ? m[g] : mw[g];
                                }
                                // An atom is never its own neighbour: its candidate at the
                                // zero offset (staged position ks) is cleared once per block
                                // instead of being tested in every chunk.
#pragma unroll
                                for (int g = 0; g < GROUP; g++) {
                                    if (ks[g] >= 0 && lane == (ks[g] >> 5) - cb)
                                        mw[g] &= ~(1u << (ks[g] & 31));
                                }
#pragma unroll
                                for (int g = 0; g < GROUP; g++)
                                    cnt[g] += (int)__reduce_add_sync(full, (unsigned)__popc(mw[g]));
                                if (mbase >= 0 && lane < ce - cb) {
                                    const long long w0 = mbase + (kb >> 5) + cb + lane;
#pragma unroll
                                    for (int g = 0; g < GROUP; g++) {
                                        if (g0 + g < ni &&
                                            !word_bad(a, w0 + (long long)(g0 + g) * nchunks_all))
                                            a.mask_pool[w0 + (long long)(g0 + g) * nchunks_all] =
                                                mw[g];
                                    }
                                }
                            }
                            if (lane < GROUP && g0 + lane < ni) {
                                int cg = cnt[0];
#pragma unroll
                                for (int g = 1; g < GROUP; g++)
                                    if (lane == g) cg = cnt[g];
                                sm.icount[g0 + lane] += cg;
                            }
                            __syncwarp();
                        }
                    } else {
                        for (int il = 0; il < ni; il++) {
                            const int si = sm.isi[il];
                            const float4 pi32 = sm.i32[il];
                            const double4 pi64 = a.pos64[si];
                            const int kself_tile = kself0 + si - kb;
                            int cnt = 0;
                            unsigned mword = 0;
                            for (int ch = 0; ch < nck; ch++) {
                                const unsigned mask = chunk_mask<FP32, KIND, RUN>(
                                    sm.cand, sm.sg, a, H, RUN ? c.S : nullptr, nseg, kb, ch * 32, lane,
                                    kself_tile, si, pi32, pi64, 0);
                                cnt += __popc(mask);
                                mword = (lane == (ch & 31)) ? mask : mword;
                                if (mbase >= 0 && ((ch & 31) == 31 || ch == nck - 1)) {
                                    const long long wi = mbase + (long long)il * nchunks_all +
                                                         (kb >> 5) + (ch & ~31) + lane;
                                    if (lane <= (ch & 31) && !word_bad(a, wi))
                                        a.mask_pool[wi] = mword;
                                }
                            }
                            if (lane == 0) sm.icount[il] += cnt;
                            __syncwarp();
                        }
                    }
                }
            }
            if (lane < ni &&
                !checked_fail(sm.iatom[lane] < 0 || sm.iatom[lane] >= a.natoms, a.err))
                a.counts[sm.iatom[lane]] = sm.icount[lane];
            __syncwarp();
        } while (0);
        L.step();
    }
}

template <bool FP32, int KIND, int GROUP, int WARPS, int CAND, bool RUN>
__global__ void __launch_bounds__(WARPS * 32, count_min_blocks(WARPS))
k_count(TraverseArgs a) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    const int warp = threadIdx.x >> 5;
    count_items<FP32, KIND, GROUP, CAND, RUN>(a, dyn_smem, blockIdx.x * WARPS + warp,
                                              gridDim.x * WARPS);
}

// Segment of candidate kk of the batch: from the table, else by search.
template <bool FP32>
__device__ __forceinline__ int seg_of_tab(const FillSmem<FP32> &sm, int nseg, int kk) {
    return kk < kCandTab ? (int)sm.cand_seg[kk] : seg_of(sm.sg, nseg, kk);
}

// One output pair in flight: where it goes and the j-side data it needs.
struct PairWork {
    bool act;
    int il, seg;
    long long slot;
    double4 pj;
    int4 aj;
};

// Map window position P to its pair and issue the j-side loads.
template <bool FP32>
__device__ __forceinline__ PairWork fetch_pair(const FillSmem<FP32> &sm,
                                               const TraverseArgs &a, int nseg, int nchunks,
                                               int nw, int nch, float inv_nch, int kr,
                                               int a0, int total_w, int P, bool tab) {
    PairWork w;
    w.act = P < total_w;
    w.il = 0;
    w.seg = 0;
    w.slot = 0;
    if (w.act) {
        int al, kk;
        if (tab) {
            const uint32_t e = sm.ptab[P];
            al = (int)(e >> 13);
            kk = kr + (int)(e & 8191u);
        } else {
            int lo = 0, hi = nw - 1;  // last word with mpre <= P
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (sm.mpre[mid] <= P)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            const int bit = nth_set_bit(sm.mw[lo], P - sm.mpre[lo]);
            al = div_small(lo, nch, inv_nch);
            kk = kr + (lo - al * nch) * 32 + bit;
        }
        w.il = a0 + al;
        w.slot = sm.abase[al] + P;
        w.seg = seg_of_tab(sm, nseg, kk);
        const int32_t sj = sm.sg.rec[w.seg].bj + kk;
        if (checked_fail(sj < 0 || sj >= a.natoms, a.err)) {
            w.act = false;
            return w;
        }
        w.pj = a.pos64[sj];
        w.aj = a.aux[sj];
    }
    return w;
}

// A pair's segment values: the segment's own offset vector (single-cell
// items) or, in a run, the one of the pair's cell offset from atom il's own
// home cell (entry v of the system's 27 visited offsets, z/y/x order).
template <bool FP32, bool RUN>
__device__ __forceinline__ SegVals pair_seg_vals(const FillSmem<FP32> &sm,
                                                 const TraverseArgs &a, const Hot &H, int seg,
                                                 int il) {
    SegVals g = seg_vals(sm.sg.rec[seg]);
    if (RUN && H.vrun >= 0) {
        // hits lie within one cell of the atom's own along x, so v < 27;
        // the clamp only keeps the table read in bounds
        int v = (int)sm.sg.row[seg] * 3 + ((int)sm.sg.xo[seg] - (int)sm.ht[il] + 1);
        checked_fail(v < 0 || v >= 27, a.err);
        v = min(max(v, 0), 26);
        const double *o = a.visit[H.vrun + v].off;
        g.o0 = o[0];
        g.o1 = o[1];
        g.o2 = o[2];
    }
    return g;
}

// Compute and store one pair (exact FP64 D and d, S, i, j).  ALL5: all five
// outputs requested and no neighbour matrix (no per-pair output checks).
// check: test the slot against the output capacity (warp-uniform; false when
// the whole list is known to fit).
template <bool FP32, bool ALL5, bool RUN>
__device__ __forceinline__ void store_pair(const FillSmem<FP32> &sm, const TraverseArgs &a,
                                           const Hot &H, const PairWork &w, bool check) {
    if (!w.act) return;
    const double4 pi = sm.i64[w.il];
    const int4 ai = sm.iaux[w.il];
    if constexpr (kChecked) {  // the slot lies in its own row
        if (checked_fail(ai.x < 0 || ai.x >= a.natoms, a.err)) return;
        if (checked_fail(w.slot < (long long)a.offsets[ai.x] ||
                             w.slot >= (long long)a.offsets[ai.x + 1],
                         a.err))
            return;
    }
    const SegVals g = pair_seg_vals<FP32, RUN>(sm, a, H, w.seg, w.il);
    const double dx = dadd(dsub(w.pj.x, pi.x), g.o0);
    const double dy = dadd(dsub(w.pj.y, pi.y), g.o1);
    const double dz = dadd(dsub(w.pj.z, pi.z), g.o2);
    const int32_t jl = (int32_t)(w.aj.x - H.atom_base);
    if (!ALL5 && a.mat_k > 0) {
        const long long rank = w.slot - (long long)a.offsets[ai.x];
        if (rank < a.mat_k) {
            const long long m = (long long)ai.x * a.mat_k + rank;
            a.mat_idx[m] = jl;
            a.mat_dist[3 * m + 0] = dx;
            a.mat_dist[3 * m + 1] = dy;
            a.mat_dist[3 * m + 2] = dz;
        }
        return;
    }
    const long long slot = w.slot;
    if (check && slot >= a.capacity) {
        atomicOr(a.err, kErrCapacity);
        return;
    }
    if (ALL5 || a.first) __stcs(a.first + slot, (int32_t)(ai.x - H.atom_base));
    if (ALL5 || a.second) __stcs(a.second + slot, jl);
    if (ALL5 || a.absdist) {
        const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
        __stcs(a.absdist + slot, __dsqrt_rn(r2));
    }
    if (ALL5 || a.distvec) {
        double *D = a.distvec + 3 * slot;
        __stcs(D, dx);
        __stcs(D + 1, dy);
        __stcs(D + 2, dz);
    }
    if (ALL5 || a.shift) {
        int32_t *Sv = a.shift + 3 * slot;
        __stcs(Sv, ai.y - ((H.pbc_bits & 1) ? w.aj.y : 0) + g.m0);
        __stcs(Sv + 1, ai.z - ((H.pbc_bits & 2) ? w.aj.z : 0) + g.m1);
        __stcs(Sv + 2, ai.w - ((H.pbc_bits & 4) ? w.aj.w : 0) + g.m2);
    }
}

// Force sink: one round of pairs, all 32 lanes.  Each active lane forms its
// pair's Lennard-Jones force on atom i from the exact FP64 D (the reference's
// operation order, as the stored D), U = 4 eps ((sigma/r)^12 - (sigma/r)^6)
// cut at the list's cutoff, F_i = -24 eps s6 (2 s6 - 1) D / r^2 with
// s6 = (sigma^2 / r^2)^3 (lj_langevin_gpu.cu:59-74 with eps = sigma = 1); the
// lanes' forces and energy shares (1/2 U per directed pair) are summed per
// atom (runs of equal i are contiguous) and the run's last lane adds them to
// the tile's shared-memory sums.
template <bool FP32, bool RUN>
__device__ __forceinline__ void lj_round(const FillSmem<FP32> &sm, double (*facc)[4],
                                         const TraverseArgs &a, const Hot &H, const PairWork &w,
                                         int lane) {
    const unsigned full = 0xffffffffu;
    double f0 = 0.0, f1 = 0.0, f2 = 0.0, e = 0.0;
    const int il = w.act ? w.il : -1;
    if (w.act) {
        const double4 pi = sm.i64[w.il];
        const SegVals g = pair_seg_vals<FP32, RUN>(sm, a, H, w.seg, w.il);
        const double dx = dadd(dsub(w.pj.x, pi.x), g.o0);
        const double dy = dadd(dsub(w.pj.y, pi.y), g.o1);
        const double dz = dadd(dsub(w.pj.z, pi.z), g.o2);
        const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
        const double ir2 = 1.0 / r2;
        const double s2 = a.lj_sig2 * ir2;
        const double s6 = s2 * s2 * s2;
        const double coef = -a.lj_eps24 * ir2 * s6 * (2.0 * s6 - 1.0);
        f0 = coef * dx;
        f1 = coef * dy;
        f2 = coef * dz;
        e = 0.5 * a.lj_eps4 * (s6 * s6 - s6);
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const double t0 = __shfl_up_sync(full, f0, d);
        const double t1 = __shfl_up_sync(full, f1, d);
        const double t2 = __shfl_up_sync(full, f2, d);
        const double t3 = __shfl_up_sync(full, e, d);
        const int ii = __shfl_up_sync(full, il, d);
        if (lane >= d && ii == il) {
            f0 += t0;
            f1 += t1;
            f2 += t2;
            e += t3;
        }
    }
    const int inext = __shfl_down_sync(full, il, 1);
    if (il >= 0 && (lane == 31 || inext != il)) {
        facc[il][0] += f0;
        facc[il][1] += f1;
        facc[il][2] += f2;
        facc[il][3] += e;
    }
    __syncwarp();
}

template <bool FP32, int KIND, bool LJ, bool ALL5, int WARPS, bool RUN>
__global__ void __launch_bounds__(WARPS * 32, fill_min_blocks(WARPS))
k_fill(TraverseArgs a) {
    constexpr int kCand = FillTile<FP32>::kCand;
    constexpr int kWarps = WARPS;
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    FillSmem<FP32> *smem = reinterpret_cast<FillSmem<FP32> *>(dyn_smem);
    // force sink: each warp's tile force and energy sums, after the warps' state
    double(*facc_all)[4] =
        reinterpret_cast<double(*)[4]>(dyn_smem + sizeof(FillSmem<FP32>) * WARPS);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    FillSmem<FP32> &sm = smem[warp];
    double(*facc)[4] = facc_all + (LJ ? warp * kITile : 0);
    const unsigned full = 0xffffffffu;
    const int nitems = *a.n_items;
    const int gwarp = blockIdx.x * kWarps + warp, nwarps = gridDim.x * kWarps;

    const bool all_rows = all_rows_of(a);
    // every slot of the list is below the output capacity: no per-pair test
    const bool cap_ok = a.offsets[a.natoms] <= a.capacity;
    ItemLoop L(a, gwarp, nitems, lane, true);
    while (L.it < nitems) {
        L.prefetch(a, nwarps, nitems, lane, true);
        const int it = L.it;
        const Home c = load_home<FP32, RUN>(a, L.rec);
        const Hot &H = c.H;

        do {
            const int ib = L.rec.ib;
            if (item_bad(a, L.rec)) break;
            int ni;
            // A run: each atom's home cell (a pair's D uses the offset of its
            // atom's own cell).
            int t_l = 0;
            if (c.run > 1) t_l = run_home_of(a, L.rec, ib + lane, lane);
            // The tile's atoms: with all rows copied asynchronously (they land
            // during the segment set-up; the row starts follow once their
            // indices are in), else the in-range ones compacted in order.
            long long my_off = 0;
            bool off_pending = false;
            if (all_rows) {
                ni = L.rec.nt;
                if (lane < ni) {
                    const char *src = reinterpret_cast<const char *>(a.pos64 + ib + lane);
                    char *dst = reinterpret_cast<char *>(&sm.i64[lane]);
                    cp_async16(dst, src);
                    cp_async16(dst + 16, src + 16);
                    cp_async16(&sm.iaux[lane], &a.aux[ib + lane]);
                    sm.isi[lane] = ib + lane;
                    sm.ht[lane] = (int8_t)t_l;
                    if (LJ) facc[lane][0] = facc[lane][1] = facc[lane][2] = facc[lane][3] = 0.0;
                }
                off_pending = true;
            } else {
                const int nt = L.rec.nt;
                int4 ax = make_int4(0, 0, 0, 0);
                bool in = false;
                if (lane < nt) {
                    ax = a.aux[ib + lane];
                    in = ax.x >= a.i_lo && ax.x < a.i_hi;
                }
                const unsigned im = __ballot_sync(full, in);
                ni = __popc(im);
                if (in) {
                    const int c2 = __popc(im & lanemask_lt());
                    const int si = ib + lane;
                    sm.i64[c2] = a.pos64[si];
                    sm.iaux[c2] = ax;
                    sm.isi[c2] = si;
                    sm.ht[c2] = (int8_t)t_l;
                    sm.icur[c2] = checked_fail(ax.x >= a.natoms, a.err)
                                      ? 0ll
                                      : (long long)a.offsets[ax.x];
                    if (LJ) facc[c2][0] = facc[c2][1] = facc[c2][2] = facc[c2][3] = 0.0;
                }
                __syncwarp();
            }
            if (ni == 0) break;
            // The first segment batch's hit words, when one window holds them
            // all (the usual case), are copied asynchronously too.
            const long long mb0 = mask_ref_base(L.hm);
            const int nch0 = mask_ref_chunks(L.hm);
            const bool words0 =
                mb0 >= 0 && c.nvisit <= kSeg && ni * nch0 <= kWinWords && nch0 * 32 <= kRange;
            if (words0)
                for (int w = lane; w < ni * nch0; w += 32)
                    if (!word_bad(a, mb0 + w)) cp_async4(&sm.mw[w], &a.mask_pool[mb0 + w]);
            for (int vb = 0; vb < c.nvisit; vb += kSeg) {
                int nseg, total, zs;
                setup_segments(sm.sg, a, c, vb, lane, nseg, total, zs);
                if (vb == 0) {
                    cp_async_wait();
                    __syncwarp();
                    if (off_pending && lane < ni) {
                        const int ax = sm.iaux[lane].x;
                        my_off = checked_fail(ax < 0 || ax >= a.natoms, a.err)
                                     ? 0ll
                                     : (long long)a.offsets[ax];
                    }
                }
                const int nchunks = (total + 31) >> 5;
                const long long mbase =
                    (a.mask_pool != nullptr && vb / kSeg < kMaskBatches)
                        ? mask_ref_base(vb == 0 ? L.hm
                                                : a.home_mask[(long long)it * kMaskBatches + vb / kSeg])
                        : -1ll;
                // segment of each tabled candidate: lane = segment
                if (lane < nseg) {
                    const int e = min(sm.sg.pref[lane + 1], kCandTab);
                    for (int k = sm.sg.pref[lane]; k < e; k++) sm.cand_seg[k] = (uint8_t)lane;
                }
                __syncwarp();
                const int kself0 = (zs >= 0) ? sm.sg.pref[zs] - sm.sg.b[zs] : INT_MIN / 2;

                for (int kr = 0; kr < total; kr += kRange) {
                    const int nrange = min(kRange, total - kr);
                    const int nch = (nrange + 31) >> 5;
                    const float inv_nch = 1.0f / (float)nch;
                    const int win = max(1, kWinWords / nch);
                    for (int a0 = 0; a0 < ni;) {
                        int na = min(win, ni - a0);
                        int nw = na * nch;
                        // --- the window's hit words ---------------------------------
                        if (mbase >= 0 && vb == 0 && kr == 0 && a0 == 0 && words0 &&
                            nch0 == nchunks) {
                            // already in shared memory (copied at the item's start)
                        } else if (mbase >= 0) {
                            for (int w = lane; w < nw; w += 32) {
                                const int al = div_small(w, nch, inv_nch);
                                const long long wi = mbase + (long long)(a0 + al) * nchunks +
                                                     (kr >> 5) + (w - al * nch);
                                sm.mw[w] = word_bad(a, wi) ? 0u : a.mask_pool[wi];
                            }
                        } else {
                            for (int kt = 0; kt < nrange; kt += kCand) {
                                const int nk = min(kCand, nrange - kt);
                                const int nkp = (nk + 31) & ~31;
                                stage_segs<FP32>(sm.cand, sm.sg, a, nseg, kr + kt, nk, nkp, lane);
                                for (int al = 0; al < na; al++) {
                                    const int il = a0 + al, si = sm.isi[il];
                                    float4 pi32 = a.pos32[si];
                                    const double4 pi64 = sm.i64[il];
                                    int ks0 = kself0;
                                    if (c.run > 1) {  // the run's frame and the atom's own cell
                                        const float3 fo = run_frame32(*c.S, sm.ht[il]);
                                        pi32.x += fo.x;
                                        pi32.y += fo.y;
                                        pi32.z += fo.z;
                                        ks0 = run_self_base(sm.sg, c.run, vb, nseg, sm.ht[il]);
                                    }
                                    const int kself_tile = ks0 + si - (kr + kt);
                                    for (int ch = 0; ch < (nkp >> 5); ch++) {
                                        const unsigned mask = chunk_mask<FP32, KIND, RUN>(
                                            sm.cand, sm.sg, a, H, RUN ? c.S : nullptr, nseg,
                                            kr + kt, ch * 32, lane, kself_tile, si, pi32, pi64,
                                            RUN ? (int)sm.ht[il] : 0);
                                        if (lane == 0) sm.mw[al * nch + (kt >> 5) + ch] = mask;
                                    }
                                }
                            }
                        }
                        __syncwarp();
                        // --- prefix of the words' popcounts ---------------------------
                        int carry = 0;
                        for (int w0 = 0; w0 < nw; w0 += 32) {
                            const int w = w0 + lane;
                            const int p = (w < nw) ? __popc(sm.mw[w]) : 0;
                            int incl = p;
#pragma unroll
                            for (int d = 1; d < 32; d <<= 1) {
                                const int o = __shfl_up_sync(full, incl, d);
                                if (lane >= d) incl += o;
                            }
                            if (w < nw) sm.mpre[w] = carry + incl - p;
                            carry += __shfl_sync(full, incl, 31);
                        }
                        if (lane == 0) sm.mpre[nw] = carry;
                        __syncwarp();
                        // --- a window over the position table keeps only the atoms
                        //     whose pairs fit it (at least one); the next window
                        //     starts at the first atom left out ---------------------
                        if (carry > kPosTab && na > 1) {
                            const bool fits = lane >= 1 && lane <= na &&
                                              sm.mpre[lane * nch] <= kPosTab;
                            na = max(1, __popc(__ballot_sync(full, fits)));
                            nw = na * nch;
                            carry = sm.mpre[nw];
                        }
                        if (off_pending) {  // the row starts loaded after the tile landed
                            if (lane < ni) sm.icur[lane] = my_off;
                            off_pending = false;
                            __syncwarp();
                        }
                        // per-atom output base: slot = abase[atom] + window position
                        if (lane < na) sm.abase[lane] = sm.icur[a0 + lane] - sm.mpre[lane * nch];
                        __syncwarp();
                        // --- small windows: each word writes its bits' positions into
                        //     a table (lane = word, ffs over its set bits), so a lane
                        //     finds its pair with one shared-memory load --------------
                        const bool tab = carry <= kPosTab;
                        if (tab) {
                            for (int w = lane; w < nw; w += 32) {
                                unsigned word = sm.mw[w];
                                int pos = sm.mpre[w];
                                const int al = div_small(w, nch, inv_nch);
                                const uint32_t base =
                                    (uint32_t)((w - al * nch) * 32) | ((uint32_t)al << 13);
                                while (word) {
                                    const int b = __ffs(word) - 1;
                                    word &= word - 1u;
                                    sm.ptab[pos++] = base | (uint32_t)b;
                                }
                            }
                            __syncwarp();
                        }
                        // --- emission, software-pipelined: the next round's j-side
                        //     loads are in flight while the current round computes ----
                        PairWork cur = fetch_pair<FP32>(sm, a, nseg, nchunks, nw, nch,
                                                        inv_nch, kr, a0, carry, lane, tab);
                        for (int P0 = 0; P0 < carry; P0 += 32) {
                            const PairWork nxt = fetch_pair<FP32>(sm, a, nseg, nchunks, nw,
                                                                  nch, inv_nch, kr, a0, carry,
                                                                  P0 + 32 + lane, tab);
                            if (LJ)
                                lj_round<FP32, RUN>(sm, facc, a, H, cur, lane);
                            else
                                store_pair<FP32, ALL5, RUN>(sm, a, H, cur, !cap_ok);
                            cur = nxt;
                        }
                        __syncwarp();
                        if (lane < na)
                            sm.icur[a0 + lane] += sm.mpre[(lane + 1) * nch] - sm.mpre[lane * nch];
                        __syncwarp();
                        a0 += na;
                    }
                }
            }
            if (off_pending) {  // no window ran (no candidates)
                if (lane < ni) sm.icur[lane] = my_off;
                __syncwarp();
            }
            // --- fill must land exactly on the next row; matrix row lengths --------
            if (lane < ni && !checked_fail(sm.iaux[lane].x < 0 ||
                                               sm.iaux[lane].x >= a.natoms, a.err)) {
                const int ax = sm.iaux[lane].x;
                const long long end = (long long)a.offsets[ax + 1];
                if (sm.icur[lane] != end) atomicOr(a.err, kErrInternal);
                if (a.mat_k > 0) {
                    const long long deg = end - (long long)a.offsets[ax];
                    a.mat_count[ax] = (int32_t)deg;
                    if (deg > a.mat_k) atomicOr(a.mat_overflow, 1);
                }
                if (LJ) {
                    a.lj_force[3 * (long long)ax + 0] = facc[lane][0];
                    a.lj_force[3 * (long long)ax + 1] = facc[lane][1];
                    a.lj_force[3 * (long long)ax + 2] = facc[lane][2];
                    a.lj_energy[ax] = facc[lane][3];
                }
            }
            __syncwarp();
        } while (0);
        L.step();
    }
}

// Dynamic shared memory of one CTA of each pass.
template <bool FP32, int CAND>
constexpr size_t count_smem_bytes(int warps) {
    return sizeof(CountSmem<FP32, CAND>) * (size_t)warps;
}
template <bool FP32>
constexpr size_t fill_smem_bytes(int warps, bool lj) {
    return sizeof(FillSmem<FP32>) * (size_t)warps +
           (lj ? sizeof(double) * 4 * kITile * (size_t)warps : sizeof(double) * 4);
}

using TravKernel = void (*)(TraverseArgs);

// Lets `kern` use more than 48 KB of dynamic shared memory on the current
// device (once per kernel and device; before its first launch or occupancy
// query).
inline cudaError_t prepare_kernel(TravKernel kern, size_t smem) {
    if (smem <= 48 * 1024) return cudaSuccess;
    static std::mutex mu;
    static std::set<std::pair<const void *, int>> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    if (done.count({(const void *)kern, dev})) return cudaSuccess;
    e = cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e == cudaSuccess) done.insert({(const void *)kern, dev});
    return e;
}

inline cudaError_t launch_kernel(TravKernel kern, size_t smem, int warps, const TraverseArgs &a,
                                 int grid, cudaStream_t st) {
    cudaError_t e = prepare_kernel(kern, smem);
    if (e != cudaSuccess) return e;
    if (a.item_next != nullptr && !a.ticket_ready) {
        e = cudaMemsetAsync(a.item_next, 0, sizeof(int), st);
        if (e != cudaSuccess) return e;
    }
    kern<<<grid, warps * 32, smem, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

inline int occupancy_kernel(TravKernel kern, size_t smem, int warps) {
    int n = 0;
    if (prepare_kernel(kern, smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, warps * 32, smem) !=
            cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

}  // namespace
}  // namespace nbl
