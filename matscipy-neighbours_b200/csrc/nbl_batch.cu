// nbl_batch.cu -- many independent systems in one launch sequence.
//
// A batch concatenates the atoms of its systems; every kernel of the pipeline
// runs once for the whole batch (systems are told apart by their atom range and
// their own grid definition, SysDev).  nbl_batch_setup plans the systems on the
// host, uploads every table once and sizes the outputs; nbl_batch_run then only
// enqueues memsets and kernels -- no host synchronisation, no allocation -- so
// it can be captured once into a CUDA graph (nbl_batch_capture) and replayed
// each step (nbl_batch_launch) while positions change in place.  The fill
// writes at most `capacity` pairs and flags an overflow that nbl_batch_finish
// reports (with the true count, so the caller can set up a larger batch).
//
// Autotuner: the pair passes' launch configuration is timed on the batch
// itself at set-up, each candidate configuration as the median of five runs:
//   * atoms per work item (the cell-occupancy tile): 32 or 16;
//   * count pass: block size (2, 4 or 8 warps), candidates staged per warp
//     (384 or 768 FP32 positions; 192 or 384 FP64), atoms per FP32 sweep
//     (2 or 4), then its grid (1, 2 or 4 waves of its resident CTAs) and
//     work items by atomic ticket or by fixed stride;
//   * fill pass: block size, then grid and tickets.
// The search is staged (shape first at two waves with tickets, then the grid
// for the best shape) for each tile size, and the tile size with the lower
// count + fill time wins.  The choice is cached per (SM count, cutoff kind,
// precision, atoms-per-cell bucket, visited-cells bucket), in memory and, when
// NBL_TUNE_CACHE names a file, on disk.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "nbl_b200.h"
#include "nbl_build.cuh"
#include "nbl_internal.cuh"
#include "nbl_plan.hh"

namespace nbl {

namespace {

__global__ void k_sys_offsets(const int64_t *__restrict__ offsets,
                              const int64_t *__restrict__ atom_base, int nsys,
                              int64_t natoms, int64_t *__restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s > nsys) return;
    out[s] = offsets[s < nsys ? atom_base[s] : natoms];
}

struct TuneChoice {
    int count_mult = 0, count_group = 4, fill_mult = 0, count_tickets = 1, fill_tickets = 1;
    int count_warps = 4, count_cand = 0, fill_warps = 8, itile = 32;
    float count_ms = 0.f, fill_ms = 0.f;
};

std::mutex g_tune_mutex;
std::map<std::string, TuneChoice> g_tune_cache;
bool g_tune_loaded = false;

void tune_load_locked() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char *path = std::getenv("NBL_TUNE_CACHE");
    if (!path) return;
    FILE *f = std::fopen(path, "r");
    if (!f) return;
    char key[256];
    TuneChoice c;
    while (std::fscanf(f, "%255s %d %d %d %d %d %d %d %d %d %f %f", key, &c.count_mult,
                       &c.count_group, &c.fill_mult, &c.count_tickets, &c.fill_tickets,
                       &c.count_warps, &c.count_cand, &c.fill_warps, &c.itile, &c.count_ms,
                       &c.fill_ms) == 12)
        g_tune_cache[key] = c;
    std::fclose(f);
}

void tune_store_locked(const std::string &key, const TuneChoice &c) {
    g_tune_cache[key] = c;
    const char *path = std::getenv("NBL_TUNE_CACHE");
    if (!path) return;
    FILE *f = std::fopen(path, "a");
    if (!f) return;
    std::fprintf(f, "%s %d %d %d %d %d %d %d %d %d %.6f %.6f\n", key.c_str(), c.count_mult,
                 c.count_group, c.fill_mult, c.count_tickets, c.fill_tickets, c.count_warps,
                 c.count_cand, c.fill_warps, c.itile, c.count_ms, c.fill_ms);
    std::fclose(f);
}

int bucket_log2(double v) { return v <= 1.0 ? 0 : (int)std::floor(std::log2(v)); }

}  // namespace

nbl_status set_error(nbl_status st, const char *fmt, ...);
nbl_status cuda_status(cudaError_t e, const char *where);

}  // namespace nbl

using namespace nbl;

#define NBL_CUDA(call, where)                                  \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_status(e_, where);  \
    } while (0)

struct nbl_batch {
    Plan p;
    Batch b;
    int quantities = 0;
    int64_t capacity = 0;
    void *out_base = nullptr;
    nbl_batch_outputs outs{};
    double *own_pos = nullptr;
    double *own_per_atom = nullptr;
    int32_t *own_types = nullptr;
    cudaStream_t own_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool ready = false;
    std::string tune_key;
    float tuned_count_ms = 0.f;
    float tuned_fill_ms = 0.f;
};

namespace {

struct Guard {
    int prev = -1;
    explicit Guard(int dev) {
        int cur = 0;
        if (cudaGetDevice(&cur) == cudaSuccess && dev >= 0 && dev != cur) {
            if (cudaSetDevice(dev) == cudaSuccess) prev = cur;
        }
    }
    ~Guard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

void release_outputs(nbl_batch *bt) {
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    bt->exec = nullptr;
    bt->graph = nullptr;
    if (bt->out_base) cudaFree(bt->out_base);
    bt->out_base = nullptr;
    std::memset(&bt->outs, 0, sizeof(bt->outs));
    if (bt->own_pos) cudaFree(bt->own_pos);
    if (bt->own_per_atom) cudaFree(bt->own_per_atom);
    if (bt->own_types) cudaFree(bt->own_types);
    bt->own_pos = nullptr;
    bt->own_per_atom = nullptr;
    bt->own_types = nullptr;
    bt->ready = false;
}

nbl_status batch_plan(const nbl_batch_request *req, Batch &b) {
    if (!req || req->nsys < 0 || (req->nsys > 0 && !req->systems))
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "bad batch request");
    if (req->quantities & ~31)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "Unsupported quantity specified.");
    if (req->precision != NBL_PRECISION_FP32_FILTER && req->precision != NBL_PRECISION_FP64)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "unknown precision");
    b = Batch();
    int kind = kCutScalar;
    if (req->per_atom_cutoff)
        kind = kCutPerAtom;
    else if (req->per_type_cutoff_sq && req->types)
        kind = kCutPerType;
    int64_t base = 0;
    for (int s = 0; s < req->nsys; s++) {
        const nbl_system &q = req->systems[s];
        if (q.nat < 0 || !q.cell_origin || !q.cell || !q.inv_cell || !q.pbc)
            return set_error(NBL_ERROR_INVALID_ARGUMENT, "system %d: bad geometry", s);
        SysDev S;
        int64_t ncells = 0;
        nbl_status st = plan_system(q.cell_origin, q.cell, q.inv_cell, q.pbc, q.cutoff, S,
                                    ncells);
        if (st != NBL_SUCCESS) return st;
        S.nat = (int32_t)q.nat;
        S.atom_base = base;
        S.cutoff_kind = kind;
        if (kind == kCutPerType) {
            S.ncutoffs = req->ncutoffs;
            S.pt_base = 0;
        }
        base += q.nat;
        b.sys.push_back(S);
        b.ncells.push_back(ncells);
    }
    if (kind == kCutPerType)
        b.pt64.assign(req->per_type_cutoff_sq,
                      req->per_type_cutoff_sq + (size_t)req->ncutoffs * req->ncutoffs);
    b.natoms = base;
    b.positions = req->positions;
    b.pos_on_device = req->positions_on_device != 0;
    b.per_atom = kind == kCutPerAtom ? req->per_atom_cutoff : nullptr;
    b.types = kind == kCutPerType ? req->types : nullptr;
    b.aux_on_device = req->aux_on_device != 0;
    b.fp32 = req->precision == NBL_PRECISION_FP32_FILTER;
    b.quantities = req->quantities;
    if (base > 0 && !req->positions)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "missing positions");
    return finish_batch(b, req->grid);
}

constexpr int kTuneRuns = 5;

float median_ms(std::vector<float> &v) {
    std::sort(v.begin(), v.end());
    return v.empty() ? 1e30f : v[v.size() / 2];
}

// Median device time (ms) of kTuneRuns count phases with the current launch
// configuration; 1e30 if a launch fails.
float time_count(nbl_batch *bt, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1) {
    std::vector<float> ms;
    for (int r = 0; r < kTuneRuns; r++) {
        cudaEventRecord(e0, st);
        if (enqueue_count(bt->p, bt->b, st) != NBL_SUCCESS) return 1e30f;
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) return 1e30f;
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        ms.push_back(t);
    }
    return median_ms(ms);
}

float time_fill(nbl_batch *bt, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1) {
    std::vector<float> ms;
    nbl_outputs o{bt->outs.first, bt->outs.second, bt->outs.distvec, bt->outs.absdist,
                  bt->outs.shift};
    for (int r = 0; r < kTuneRuns; r++) {
        cudaEventRecord(e0, st);
        if (run_fill(bt->p, o, bt->capacity, st) != NBL_SUCCESS) return 1e30f;
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) return 1e30f;
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        ms.push_back(t);
    }
    return median_ms(ms);
}

void apply_choice(Plan &p, const TuneChoice &c) {
    p.count_mult = c.count_mult;
    p.fill_mult = c.fill_mult;
    p.count_tickets = c.count_tickets != 0;
    p.fill_tickets = c.fill_tickets != 0;
    p.count_shape.warps = c.count_warps;
    p.count_shape.cand = c.count_cand;
    p.count_shape.group = c.count_group;
    p.fill_shape.warps = c.fill_warps;
    p.itile = c.itile;
    p.itile_auto = false;
}

// Fill grid for `mult` CTAs per SM (the cap nbl_count's planning applies).
int fill_grid_of(const Plan &p, int64_t natoms, int mult) {
    return std::max(1, std::min(p.num_sms * mult, (int)std::max<int64_t>((natoms + 3) / 4, 1)));
}

// The best count and fill configuration for one tile size; false on error.
bool tune_for_tile(nbl_batch *bt, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1, int itile,
                   TuneChoice &best) {
    const Batch &b = bt->b;
    Plan &p = bt->p;
    const int kind = b.sys.empty() ? kCutScalar : b.sys[0].cutoff_kind;
    TuneChoice c = best;
    c.itile = itile;
    apply_choice(p, c);
    // count: shape at two waves with tickets, then the grid for the best shape
    float best_ms = 1e30f;
    const int warps[] = {2, 4, 8};
    const int groups[] = {2, 4};
    for (int w : warps) {
        for (int cand = 0; cand <= 1; cand++) {
            for (int g : groups) {
                if (!b.fp32 && g != 4) continue;  // the group only shapes the FP32 sweep
                TravShape sh;
                sh.warps = w;
                sh.cand = cand;
                sh.group = g;
                const int occ = traverse_blocks_per_sm(kModeCount, b.fp32, kind, sh);
                if (occ <= 0) continue;
                p.count_shape = sh;
                p.count_mult = 2 * occ;
                p.count_tickets = true;
                const float ms = time_count(bt, st, e0, e1);
                if (ms < best_ms) {
                    best_ms = ms;
                    c.count_warps = w;
                    c.count_cand = cand;
                    c.count_group = g;
                    c.count_mult = 2 * occ;
                    c.count_tickets = 1;
                }
            }
        }
    }
    if (best_ms >= 1e30f) return false;
    {
        TravShape sh;
        sh.warps = c.count_warps;
        sh.cand = c.count_cand;
        sh.group = c.count_group;
        p.count_shape = sh;
        const int occ = std::max(1, traverse_blocks_per_sm(kModeCount, b.fp32, kind, sh));
        const int waves[] = {1, 2, 4};
        for (int wv : waves) {
            for (int tk = 1; tk >= 0; tk--) {
                p.count_mult = wv * occ;
                p.count_tickets = tk != 0;
                const float ms = time_count(bt, st, e0, e1);
                if (ms < best_ms) {
                    best_ms = ms;
                    c.count_mult = wv * occ;
                    c.count_tickets = tk;
                }
            }
        }
    }
    c.count_ms = best_ms;
    apply_choice(p, c);
    if (enqueue_count(p, bt->b, st) != NBL_SUCCESS) return false;
    p.have_count = true;  // the fills below read this count's offsets
    // fill: block size at two waves with tickets, then the grid
    best_ms = 1e30f;
    for (int w : warps) {
        TravShape sh;
        sh.warps = w;
        const int occ = traverse_blocks_per_sm(kModeFill, b.fp32, kind, sh);
        if (occ <= 0) continue;
        p.fill_shape = sh;
        p.fill_tickets = true;
        p.fill_grid = fill_grid_of(p, b.natoms, 2 * occ);
        const float ms = time_fill(bt, st, e0, e1);
        if (ms < best_ms) {
            best_ms = ms;
            c.fill_warps = w;
            c.fill_mult = 2 * occ;
            c.fill_tickets = 1;
        }
    }
    if (best_ms >= 1e30f) return false;
    {
        TravShape sh;
        sh.warps = c.fill_warps;
        p.fill_shape = sh;
        const int occ = std::max(1, traverse_blocks_per_sm(kModeFill, b.fp32, kind, sh));
        const int waves[] = {1, 2, 4};
        for (int wv : waves) {
            for (int tk = 1; tk >= 0; tk--) {
                p.fill_tickets = tk != 0;
                p.fill_grid = fill_grid_of(p, b.natoms, wv * occ);
                const float ms = time_fill(bt, st, e0, e1);
                if (ms < best_ms) {
                    best_ms = ms;
                    c.fill_mult = wv * occ;
                    c.fill_tickets = tk;
                }
            }
        }
    }
    c.fill_ms = best_ms;
    best = c;
    return true;
}

nbl_status autotune(nbl_batch *bt, cudaStream_t st) {
    const Batch &b = bt->b;
    double cells = 0.0;
    int max_visit = 1;
    for (size_t s = 0; s < b.sys.size(); s++) {
        cells += (double)b.ncells[s];
        max_visit = std::max(max_visit, b.sys[s].nvisit);
    }
    char key[160];
    std::snprintf(key, sizeof(key), "w5_sm%d_k%d_f%d_d%d_v%d", bt->p.num_sms,
                  b.sys.empty() ? 0 : b.sys[0].cutoff_kind, b.fp32 ? 1 : 0,
                  bucket_log2(b.natoms / std::max(cells, 1.0)), bucket_log2(max_visit));
    bt->tune_key = key;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        tune_load_locked();
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            apply_choice(bt->p, it->second);
            bt->tuned_count_ms = it->second.count_ms;
            bt->tuned_fill_ms = it->second.fill_ms;
            return NBL_SUCCESS;
        }
    }
    cudaEvent_t e0, e1;
    NBL_CUDA(cudaEventCreate(&e0), "event");
    NBL_CUDA(cudaEventCreate(&e1), "event");
    TuneChoice best;
    bool have = false;
    const int tiles[] = {32, 16};
    for (int t : tiles) {
        TuneChoice c;
        if (!tune_for_tile(bt, st, e0, e1, t, c)) continue;
        if (!have || c.count_ms + c.fill_ms < best.count_ms + best.fill_ms) best = c;
        have = true;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!have) {
        apply_choice(bt->p, TuneChoice());
        return set_error(NBL_ERROR_INTERNAL, "autotuner: no launch configuration ran");
    }
    apply_choice(bt->p, best);
    bt->tuned_count_ms = best.count_ms;
    bt->tuned_fill_ms = best.fill_ms;
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    tune_store_locked(key, best);
    return NBL_SUCCESS;
}

}  // namespace

extern "C" {

NBL_API nbl_status nbl_batch_create(int device_id, nbl_batch **out) {
    if (!out) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null batch pointer");
    *out = nullptr;
    nbl_plan *tmp = nullptr;
    nbl_status st = nbl_plan_create(device_id, &tmp);  // validates the device
    if (st != NBL_SUCCESS) return st;
    nbl_plan_destroy(tmp);
    nbl_batch *bt = new (std::nothrow) nbl_batch();
    if (!bt) return set_error(NBL_ERROR_OUT_OF_MEMORY, "host allocation failed");
    int dev = device_id;
    if (dev < 0) cudaGetDevice(&dev);
    bt->p.device = dev;
    Guard g(dev);
    cudaDeviceGetAttribute(&bt->p.num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaMallocHost(&bt->p.host_small, sizeof(int64_t) * 4) != cudaSuccess ||
        cudaEventCreateWithFlags(&bt->p.stage_done, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&bt->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete bt;
        return set_error(NBL_ERROR_CUDA, "cannot create batch resources");
    }
    *out = bt;
    return NBL_SUCCESS;
}

NBL_API nbl_status nbl_batch_destroy(nbl_batch *bt) {
    if (!bt) return NBL_SUCCESS;
    Guard g(bt->p.device);
    cudaDeviceSynchronize();
    release_outputs(bt);
    bt->p.ws.release();
    if (bt->p.host_small) cudaFreeHost(bt->p.host_small);
    if (bt->p.host_stage) cudaFreeHost(bt->p.host_stage);
    if (bt->p.stage_done) cudaEventDestroy(bt->p.stage_done);
    if (bt->own_stream) cudaStreamDestroy(bt->own_stream);
    delete bt;
    return NBL_SUCCESS;
}

NBL_API nbl_status nbl_batch_setup(nbl_batch *bt, const nbl_batch_request *req,
                                   int64_t capacity) {
    if (!bt || !req) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null argument");
    Guard g(bt->p.device);
    cudaStream_t st = bt->own_stream;
    NBL_CUDA(cudaStreamSynchronize(st), "batch set-up");
    release_outputs(bt);
    nbl_status s = batch_plan(req, bt->b);
    if (s != NBL_SUCCESS) return s;
    Batch &b = bt->b;
    bt->quantities = req->quantities;
    const int64_t N = b.natoms;
    // Host inputs become batch-owned device copies (the graph reads them in place).
    if (!b.pos_on_device && N > 0) {
        NBL_CUDA(cudaMalloc((void **)&bt->own_pos, sizeof(double) * 3 * N), "positions");
        NBL_CUDA(cudaMemcpy(bt->own_pos, b.positions, sizeof(double) * 3 * N,
                            cudaMemcpyHostToDevice), "positions");
        b.positions = bt->own_pos;
        b.pos_on_device = true;
    }
    if (!b.aux_on_device && N > 0 && (b.per_atom || b.types)) {
        if (b.per_atom) {
            NBL_CUDA(cudaMalloc((void **)&bt->own_per_atom, sizeof(double) * N), "cutoffs");
            NBL_CUDA(cudaMemcpy(bt->own_per_atom, b.per_atom, sizeof(double) * N,
                                cudaMemcpyHostToDevice), "cutoffs");
            b.per_atom = bt->own_per_atom;
        }
        if (b.types) {
            NBL_CUDA(cudaMalloc((void **)&bt->own_types, sizeof(int32_t) * N), "types");
            NBL_CUDA(cudaMemcpy(bt->own_types, b.types, sizeof(int32_t) * N,
                                cudaMemcpyHostToDevice), "types");
            b.types = bt->own_types;
        }
        b.aux_on_device = true;
    }
    s = upload_batch(bt->p, b, st);
    if (s != NBL_SUCCESS) return s;
    NBL_CUDA(cudaStreamSynchronize(st), "batch upload");
    bt->p.stage_in_flight = false;
    // Capacity: measured when not given (25 % headroom for later steps).
    if (capacity <= 0) {
        s = enqueue_count(bt->p, b, st);
        if (s != NBL_SUCCESS) return s;
        NBL_CUDA(cudaMemcpyAsync(bt->p.host_small, bt->p.bufs.offsets + N,
                                 sizeof(int64_t) + sizeof(int) * 6, cudaMemcpyDeviceToHost, st),
                 "read pair count and mask demand");
        NBL_CUDA(cudaStreamSynchronize(st), "count");
        capacity = bt->p.host_small[0] + bt->p.host_small[0] / 4 + 4096;
        // More hit words asked for than the estimate held: re-plan the
        // workspace with the measured demand before the graph is captured.
        int flags[6];
        std::memcpy(flags, bt->p.host_small + 1, sizeof(flags));
        unsigned long long demand = 0;
        std::memcpy(&demand, flags + 4, sizeof(demand));
        if ((long long)demand > bt->p.bufs.mask_cap) {
            bt->p.mask_hint = (int64_t)demand;
            s = upload_batch(bt->p, b, st);
            if (s != NBL_SUCCESS) return s;
            NBL_CUDA(cudaStreamSynchronize(st), "batch upload");
            bt->p.stage_in_flight = false;
        }
    }
    bt->capacity = capacity;
    const int q = req->quantities;
    const size_t cap = (size_t)std::max<int64_t>(capacity, 1);
    size_t off[6], total = 0;
    auto add = [&](size_t bytes) {
        size_t o = total;
        total += (bytes + 255) & ~size_t(255);
        return o;
    };
    off[0] = (q & NBL_QUANTITY_FIRST) ? add(sizeof(int32_t) * cap) : 0;
    off[1] = (q & NBL_QUANTITY_SECOND) ? add(sizeof(int32_t) * cap) : 0;
    off[2] = (q & NBL_QUANTITY_DISTVEC) ? add(sizeof(double) * 3 * cap) : 0;
    off[3] = (q & NBL_QUANTITY_ABSDIST) ? add(sizeof(double) * cap) : 0;
    off[4] = (q & NBL_QUANTITY_SHIFT) ? add(sizeof(int32_t) * 3 * cap) : 0;
    off[5] = add(sizeof(int64_t) * (b.sys.size() + 1));
    NBL_CUDA(cudaMalloc(&bt->out_base, total), "batch outputs");
    char *base = static_cast<char *>(bt->out_base);
    bt->outs.first = (q & NBL_QUANTITY_FIRST) ? (int32_t *)(base + off[0]) : nullptr;
    bt->outs.second = (q & NBL_QUANTITY_SECOND) ? (int32_t *)(base + off[1]) : nullptr;
    bt->outs.distvec = (q & NBL_QUANTITY_DISTVEC) ? (double *)(base + off[2]) : nullptr;
    bt->outs.absdist = (q & NBL_QUANTITY_ABSDIST) ? (double *)(base + off[3]) : nullptr;
    bt->outs.shift = (q & NBL_QUANTITY_SHIFT) ? (int32_t *)(base + off[4]) : nullptr;
    bt->outs.sys_offsets = (int64_t *)(base + off[5]);
    bt->outs.capacity = capacity;
    bt->outs.positions = const_cast<double *>(b.positions);
    if (req->autotune) {
        s = autotune(bt, st);
        if (s != NBL_SUCCESS) return s;
        NBL_CUDA(cudaStreamSynchronize(st), "autotune");
    }
    bt->ready = true;
    return NBL_SUCCESS;
}

NBL_API nbl_status nbl_batch_run(nbl_batch *bt, void *stream) {
    if (!bt || !bt->ready) return set_error(NBL_ERROR_INVALID_ARGUMENT, "batch not set up");
    Guard g(bt->p.device);
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : bt->own_stream;
    nbl_status s = enqueue_count(bt->p, bt->b, st);
    if (s != NBL_SUCCESS) return s;
    bt->p.have_count = true;
    nbl_outputs o{bt->outs.first, bt->outs.second, bt->outs.distvec, bt->outs.absdist,
                  bt->outs.shift};
    s = run_fill(bt->p, o, bt->capacity, st);
    if (s != NBL_SUCCESS) return s;
    const int nsys = (int)bt->b.sys.size();
    k_sys_offsets<<<(nsys + 1 + 127) / 128, 128, 0, st>>>(
        bt->p.bufs.offsets, bt->p.bufs.sys_atom_base, nsys, bt->b.natoms,
        bt->outs.sys_offsets);
    count_launch();
    NBL_CUDA(cudaGetLastError(), "k_sys_offsets");
    return NBL_SUCCESS;
}

NBL_API nbl_status nbl_batch_capture(nbl_batch *bt, void *stream) {
    if (!bt || !bt->ready) return set_error(NBL_ERROR_INVALID_ARGUMENT, "batch not set up");
    Guard g(bt->p.device);
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : bt->own_stream;
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    bt->exec = nullptr;
    bt->graph = nullptr;
    NBL_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    nbl_status s = nbl_batch_run(bt, st);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (s != NBL_SUCCESS) {
        if (graph) cudaGraphDestroy(graph);
        return s;
    }
    NBL_CUDA(e, "end capture");
    bt->graph = graph;
    NBL_CUDA(cudaGraphInstantiate(&bt->exec, graph, 0), "graph instantiate");
    return NBL_SUCCESS;
}

NBL_API nbl_status nbl_batch_launch(nbl_batch *bt, void *stream) {
    if (!bt || !bt->exec) return set_error(NBL_ERROR_INVALID_ARGUMENT, "no captured graph");
    Guard g(bt->p.device);
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : bt->own_stream;
    NBL_CUDA(cudaGraphLaunch(bt->exec, st), "graph launch");
    return NBL_SUCCESS;
}

NBL_API nbl_status nbl_batch_finish(nbl_batch *bt, void *stream, int64_t *npairs) {
    if (!bt || !bt->ready || !npairs)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "batch not set up");
    Guard g(bt->p.device);
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : bt->own_stream;
    const int64_t N = bt->b.natoms;
    NBL_CUDA(cudaMemcpyAsync(bt->p.host_small, bt->p.bufs.offsets + N,
                             sizeof(int64_t) + sizeof(int) * 2, cudaMemcpyDeviceToHost, st),
             "read pair count and flags");
    NBL_CUDA(cudaStreamSynchronize(st), "batch");
    int flags[2];
    std::memcpy(flags, bt->p.host_small + 1, sizeof(flags));
    *npairs = bt->p.host_small[0];
    if (flags[1] & kErrRange)
        return set_error(NBL_ERROR_RANGE,
                         "positions must be finite and within 2^29 cells of the box");
    // an internal bound makes the pair count meaningless: report it first
    if (flags[1] & kErrInternal)
        return set_error(NBL_ERROR_INTERNAL, "device-side bound exceeded");
    if (*npairs > bt->capacity || (flags[1] & kErrCapacity))
        return set_error(NBL_ERROR_CAPACITY,
                         "%lld pairs exceed the batch capacity %lld; set up again with a "
                         "larger capacity", (long long)*npairs, (long long)bt->capacity);
    return NBL_SUCCESS;
}

NBL_API nbl_status nbl_batch_get_outputs(nbl_batch *bt, nbl_batch_outputs *out) {
    if (!bt || !bt->ready || !out)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "batch not set up");
    *out = bt->outs;
    return NBL_SUCCESS;
}

NBL_API nbl_status nbl_batch_get_config(nbl_batch *bt, int *count_mult, int *count_group,
                                        int *fill_mult) {
    if (!bt) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null batch");
    if (count_mult) *count_mult = bt->p.count_mult;
    if (count_group) *count_group = bt->p.count_shape.group;
    if (fill_mult) *fill_mult = bt->p.fill_mult;
    return NBL_SUCCESS;
}

NBL_API nbl_status nbl_batch_get_tickets(nbl_batch *bt, int *count_tickets, int *fill_tickets) {
    if (!bt) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null batch");
    if (count_tickets) *count_tickets = bt->p.count_tickets ? 1 : 0;
    if (fill_tickets) *fill_tickets = bt->p.fill_tickets ? 1 : 0;
    return NBL_SUCCESS;
}

NBL_API nbl_status nbl_batch_get_launch_config(nbl_batch *bt, nbl_launch_config *cfg,
                                               float *count_ms, float *fill_ms) {
    if (!bt || !cfg) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null argument");
    launch_config_of(bt->p, cfg);
    if (count_ms) *count_ms = bt->tuned_count_ms;
    if (fill_ms) *fill_ms = bt->tuned_fill_ms;
    return NBL_SUCCESS;
}

}  // extern "C"
