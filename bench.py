"""Benchmark: neighbour-list pairs/s on B200 for the dense-bulk configuration.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one "step" = one full neighbour_list("ijdDS") build): 1,048,576 atoms
on an FCC lattice (a = 3.6 A, 64^3 unit cells), Gaussian jitter 0.1 A, cell
sheared by xy = 0.2 Lx and xz = 0.1 Lx, periodic, cutoff 5.0 A, FP64 -- seeded
synthetic data.  Each step bins, sorts, counts, scans and fills the exact pair
list (bit-identical to the reference CPU path).

* value: pairs/s with positions resident in HBM, device time per step from
  CUDA events on the engine's stream, L2 flushed (a 256 MiB write) between
  steps outside the timed events; whole-job aggregate over ranks.
* e2e:   the same metric through the public API with host numpy buffers:
  every step copies the positions host->device and all five output arrays
  device->host (pinned host memory).
* roofline: the fill kernel (the HBM-bound pass that writes 52 B per pair),
  algorithmic bytes (npairs * 52 + nat * 24) / its CUDA-event time, against
  the measured HBM copy bandwidth.
* cpu_baseline: the reference's own CPU core (oracle/_ref, OpenMP, all host
  threads) on the same workload, rank 0 at N = 1.

Under torchrun each rank builds its own replica of the workload (seed = rank):
independent systems, no collective on the data path (weak scaling).
"""
import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "matscipy-neighbours_b200"))

WORKLOAD = {"workload": "fcc_bulk_triclinic_1M", "natoms": 1048576, "lattice": "fcc",
            "a_A": 3.6, "reps": 64, "jitter_A": 0.1, "shear": [0.2, 0.1],
            "pbc": "TTT", "cutoff_A": 5.0, "quantities": "ijdDS"}
METRIC = "pairs/s (exact pair set, dense bulk FCC 1M atoms, ijdDS)"
UNIT = "pairs/s"
BYTES_PER_PAIR = 52   # i 4 + j 4 + d 8 + D 24 + S 12
BYTES_PER_ATOM_IN = 24


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def _workloads():
    """The seeded workload generators, loaded from their own file: importing
    them through the package would run its __init__, which loads the engine's
    CUDA library, and the reference arm must run without any engine code in
    the process."""
    import importlib.util
    name = "nbl_bench_workloads"
    if name not in sys.modules:
        path = ROOT / "matscipy-neighbours_b200" / "matscipy_neighbours" / "_workloads.py"
        spec = importlib.util.spec_from_file_location(name, path)
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def _oracle():
    """The CPU checker (oracle/): the reference's own core when it was built
    (oracle/_ref), else the C restatement."""
    if str(ROOT / "oracle") not in sys.path:
        sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    return O


def _same(got, want):
    """Bit-identical arrays (floats compared by their bit patterns)."""
    import numpy as np
    got = np.asarray(got)
    want = np.asarray(want)
    if got.shape != want.shape or got.dtype != want.dtype:
        return False
    if got.dtype.kind == "f":
        return bool(np.array_equal(got.view(np.int64), want.view(np.int64)))
    return bool(np.array_equal(got, want))


def _same_device(quantities, dev_arrays, want):
    """Engine outputs (torch device tensors, one per quantity) against the
    checker's host arrays, one quantity at a time (bounded host memory)."""
    if len(quantities) == 1:
        want = (want,)
    for q, t, w in zip(quantities, dev_arrays, want):
        if not _same(t.cpu().numpy(), w):
            return False
    return True


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured", d
        except Exception:
            pass
    return 6650.0, "fallback", {}


def _traffic_per_launch(npairs, nat):
    p = ROOT / "profiles" / "fill_traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        return d["bytes_per_pair"] * npairs + d.get("bytes_per_atom", 0.0) * nat
    except Exception:
        return None


class ClockSampler:
    """SM clock and throttle reasons sampled every 20 ms during the timed region
    (read-only NVML queries; nvidia-smi as a fallback)."""

    # NVML clocks-event-reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, torch_device):
        self.dev = torch_device
        self.samples = []
        self.reasons = set()
        self.sm_max = None
        self._stop = threading.Event()
        self._thread = None
        self.handle = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            props = torch.cuda.get_device_properties(torch_device)
            bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self.sm_max = float(pynvml.nvmlDeviceGetMaxClockInfo(self.handle,
                                                                 pynvml.NVML_CLOCK_SM))
        except Exception:
            self.handle = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(float(self.nvml.nvmlDeviceGetClockInfo(
                    self.handle, self.nvml.NVML_CLOCK_SM)))
                bits = int(self.nvml.nvmlDeviceGetCurrentClocksEventReasons(self.handle))
                for b, name in self.REASONS.items():
                    if bits & b:
                        self.reasons.add(name)
            except Exception:
                pass
            self._stop.wait(0.02)

    def start(self):
        if self.handle is not None:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()

    def stop(self):
        if self._thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"],
                    "samples": 0}
        self._stop.set()
        self._thread.join(timeout=2)
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.sm_max, "reasons": sorted(self.reasons),
                "samples": len(self.samples), "source": "nvml, 20 ms"}


def _time_batch(b, steps, warmup):
    """Median device time (ms) of `steps` replays of a batch's graph, each
    bracketed by CUDA events on the batch's stream."""
    import torch
    stream = torch.cuda.current_stream(b.device)
    for _ in range(warmup):
        b.run()
    ms = []
    for _ in range(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        b.stream.wait_stream(stream)
        e0.record(b.stream)
        b.launch()
        e1.record(b.stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    b.finish()
    return statistics.median(ms)


def batched_bench(steps, warmup, dev, rank=0, check=False):
    """C4: 4,096 small systems (sizes log-uniform 8-512, random triclinic cells
    scaled towards 0.08 A^-3, random pbc, per-atom radii 3-6 A, ijdDS).
    Batched: the FP32-filter build of all systems replayed from one captured
    CUDA graph, and the same graph with the plain FP64 test (the precision
    gain alone).  Plain: one FP64 nbl_count + nbl_fill per system (the
    batching gain on top).  With `check`, every system's output is compared
    bit for bit with the CPU checker run on that system alone."""
    import ctypes

    import numpy as np
    import torch

    from matscipy_neighbours import _matscipy_neighbours as ext
    from matscipy_neighbours.batch import NeighbourListBatch
    W = _workloads()

    systems = W.batched_systems(seed=1 + rank)
    b64 = NeighbourListBatch(systems, precision="fp64", graph=True, autotune=True,
                             device=dev.index)
    fp64_ms = _time_batch(b64, steps, warmup)
    lc64 = b64.launch_config()
    b64.close()
    b = NeighbourListBatch(systems, precision="fp32", graph=True, autotune=True,
                           device=dev.index)
    stream = torch.cuda.current_stream(dev)
    batched_ms = _time_batch(b, steps, warmup)
    npairs = b.npairs
    parity = None
    if check:
        O = _oracle()
        _, _, fn = _cpu_fn(O, len(os.sched_getaffinity(0)))
        off = b.sys_offsets()
        res = [t.cpu().numpy() for t in b.results()]
        parity = True
        for s, sd in enumerate(systems):
            want = fn("ijdDS", sd["cell"], sd["positions"], sd["cutoff"], sd["pbc"])
            if not all(_same(r[off[s]:off[s + 1]], w) for r, w in zip(res, want)):
                parity = False
                break
        del res
    lc = b.launch_config()
    positions = b.positions
    offs = b.atom_offsets
    b.close()

    # plain per-system FP64 launches over the same resident positions
    plan = ext.plan_for(dev.index)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    cap = int(npairs * 1.1) + 1024
    outs = {"i": torch.empty(cap, dtype=torch.int32, device=dev),
            "j": torch.empty(cap, dtype=torch.int32, device=dev),
            "D": torch.empty((cap, 3), dtype=torch.float64, device=dev),
            "d": torch.empty(cap, dtype=torch.float64, device=dev),
            "S": torch.empty((cap, 3), dtype=torch.int32, device=dev)}
    prev = ext.set_options(precision="fp64", grid="auto")
    reqs = []
    keep = []
    for k, sd in enumerate(systems):
        cell = np.ascontiguousarray(sd["cell"])
        inv = np.ascontiguousarray(np.linalg.inv(cell.T))
        pbc8 = np.ascontiguousarray(np.asarray(sd["pbc"], dtype=np.uint8))
        rc, pa, pt, nc = ext.resolve_cutoff(np.asarray(sd["cutoff"]), len(sd["positions"]))
        origin = np.zeros(3)
        keep.extend([cell, inv, pbc8, pa, origin])
        pos_ptr = positions.data_ptr() + int(offs[k]) * 24
        reqs.append(ext.make_request(31, origin, cell, inv, pbc8, len(sd["positions"]),
                                     ctypes.c_void_p(pos_ptr), True, rc, pa, None, 0,
                                     None, dev.index))
    ext.set_options(**prev)

    def plain_pass():
        n = ctypes.c_int64()
        base = 0
        for r in reqs:
            ext.check(ext.lib.nbl_count(plan, ctypes.byref(r), sptr, ctypes.byref(n)))
            o = ext.Outputs()
            o.first = outs["i"].data_ptr() + 4 * base
            o.second = outs["j"].data_ptr() + 4 * base
            o.distvec = outs["D"].data_ptr() + 24 * base
            o.absdist = outs["d"].data_ptr() + 8 * base
            o.shift = outs["S"].data_ptr() + 12 * base
            ext.check(ext.lib.nbl_fill(plan, ctypes.byref(o), sptr))
            base += n.value
        return base

    plain_pass()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    tot = plain_pass()
    torch.cuda.synchronize(dev)
    plain_s = time.perf_counter() - t0
    assert tot == npairs, (tot, npairs)
    batched_s = batched_ms * 1e-3
    out = {"workload": "batched_4096_systems", "systems": len(systems),
           "atoms": int(offs[-1]), "npairs": int(npairs),
           "batched_fp32_graph": {"value": npairs / batched_s, "unit": UNIT,
                                  "ms_per_step": batched_ms,
                                  "stage_ms_at_tuning": {"count_phase": lc["tuned_count_ms"],
                                                         "fill": lc["tuned_fill_ms"]},
                                  "launch_config": lc},
           "batched_fp64_graph": {"value": npairs / (fp64_ms * 1e-3), "unit": UNIT,
                                  "ms_per_step": fp64_ms,
                                  "stage_ms_at_tuning": {"count_phase": lc64["tuned_count_ms"],
                                                         "fill": lc64["tuned_fill_ms"]},
                                  "launch_config": lc64},
           "plain_fp64_per_system": {"value": npairs / plain_s, "unit": UNIT,
                                     "ms_per_step": plain_s * 1e3,
                                     "note": "one nbl_count + nbl_fill per system, host "
                                             "wall clock (4,096 synchronising calls)"},
           "speedup": plain_s / batched_s,
           "speedup_precision_only": fp64_ms / batched_ms,
           "speedup_batching_only": plain_s / (fp64_ms * 1e-3)}
    if parity is not None:
        out["parity"] = parity
    return out


def configs_bench(dev, flush, reps=10, only=None, check=False, thread_per_atom=0):
    """The other configurations beside the headline (rank 0, N = 1): C1 plain
    small, C3 sparse slab (per-type cutoffs, ijdD), C5 differentiation lattice,
    and a dilute gas (200,000 atoms, 0.5 per cell).  Each: positions resident
    on the device, median of `reps` full builds (count + fill) by CUDA events
    with the L2 flushed before each, and the reference's CPU core on the same
    input (all host threads, median of 3).  C3 and the dilute gas also time
    both pair-pass forms (one warp per work item, one thread per atom).
    C5 adds the backward kernel (nbl_backward, gradients of D and d), timed
    alone, with its HBM roofline: npairs * 84 + nat * 48 algorithmic bytes.
    `thread_per_atom` is the plans' launch-config setting for every line
    (0: the default choice, 1: on, -1: off)."""
    import ctypes

    import numpy as np
    import torch

    O = _oracle()
    W = _workloads()
    from matscipy_neighbours import _matscipy_neighbours as ext
    from matscipy_neighbours.autograd import BackwardArgs, _lib

    peak, peak_kind, _ = _peaks()
    cores = len(os.sched_getaffinity(0))
    have_ref = O.ref_available()
    if have_ref:
        O.ref_set_threads(cores)
    cpu_fn = O.ref_neighbour_list if have_ref else O.oracle_neighbour_list
    stream = torch.cuda.current_stream(dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    plan = ext.plan_for(dev.index)
    out = {}
    def wanted(name):
        return only is None or name in only

    def set_passes(setting):
        cfg = ext.LaunchConfig(thread_per_atom=setting)
        ext.check(ext.lib.nbl_plan_set_launch_config(plan, ctypes.byref(cfg)))

    set_passes(thread_per_atom)
    for name, make in (("C1_plain_small", W.plain_small),
                       ("C3_sparse_slab", W.sparse_slab),
                       ("C5_diff_lattice", W.diff_lattice),
                       ("gas_dilute", W.dilute_gas)):
        if not wanted(name):
            continue
        w = make()
        q = w["quantities"]
        flags = ext.quantity_flags(q)
        nat = w["positions"].shape[0]
        cell = np.ascontiguousarray(w["cell"], dtype=float)
        inv = np.ascontiguousarray(np.linalg.inv(cell.T))
        pbc8 = np.ascontiguousarray(np.asarray(w["pbc"], dtype=np.uint8))
        origin = np.zeros(3)
        rc, pa, pt, nc = ext.resolve_cutoff(w["cutoff"], nat)
        types = w.get("numbers")
        types = None if types is None else np.ascontiguousarray(types, dtype=np.int32)
        pos = torch.from_numpy(np.ascontiguousarray(w["positions"])).to(dev)
        grids = ["auto"] + (["dense", "morton", "hashed"] if name.startswith("C3") else [])
        n = ctypes.c_int64()
        bufs = None
        grid_rows = {}
        for grid in grids:
            prev = ext.set_options(grid=grid)
            req = ext.make_request(flags, origin, cell, inv, pbc8, nat,
                                   ctypes.c_void_p(pos.data_ptr()), True, rc, pa, pt, nc,
                                   types, dev.index)
            ext.set_options(grid=prev["grid"])
            ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), sptr, ctypes.byref(n)))
            npairs = int(n.value)
            if bufs is None:
                bufs = {"i": torch.empty(npairs, dtype=torch.int32, device=dev),
                        "j": torch.empty(npairs, dtype=torch.int32, device=dev),
                        "D": torch.empty((npairs, 3), dtype=torch.float64, device=dev),
                        "d": torch.empty(npairs, dtype=torch.float64, device=dev),
                        "S": torch.empty((npairs, 3), dtype=torch.int32, device=dev)}
                o = ext._outputs_struct({c: bufs[c] for c in q}, lambda t: t.data_ptr())
            ms, cms, fms = [], [], []
            for k in range(reps + 3):
                flush.zero_()
                torch.cuda.synchronize(dev)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e2 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), sptr, ctypes.byref(n)))
                e1.record(stream)
                ext.check(ext.lib.nbl_fill(plan, ctypes.byref(o), sptr))
                e2.record(stream)
                e2.synchronize()
                if k >= 3:
                    ms.append(e0.elapsed_time(e2))
                    cms.append(e0.elapsed_time(e1))
                    fms.append(e1.elapsed_time(e2))
            ext.check(ext.lib.nbl_check(plan, sptr))
            grid_rows[grid] = (statistics.median(ms), statistics.median(cms),
                               statistics.median(fms))
        gpu_ms, count_ms, fill_ms = grid_rows["auto"]
        passes = {}
        if name.startswith(("C3", "gas")):
            # both pair-pass forms on the same input (auto grid)
            prev = ext.set_options(grid="auto")
            req = ext.make_request(flags, origin, cell, inv, pbc8, nat,
                                   ctypes.c_void_p(pos.data_ptr()), True, rc, pa, pt, nc,
                                   types, dev.index)
            ext.set_options(grid=prev["grid"])
            for form, setting in (("warp_per_item", -1), ("thread_per_atom", 1)):
                set_passes(setting)
                ms = []
                for k in range(reps + 3):
                    flush.zero_()
                    torch.cuda.synchronize(dev)
                    e0 = torch.cuda.Event(enable_timing=True)
                    e2 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), sptr,
                                                ctypes.byref(n)))
                    ext.check(ext.lib.nbl_fill(plan, ctypes.byref(o), sptr))
                    e2.record(stream)
                    e2.synchronize()
                    if k >= 3:
                        ms.append(e0.elapsed_time(e2))
                ext.check(ext.lib.nbl_check(plan, sptr))
                passes[form] = statistics.median(ms)
            set_passes(thread_per_atom)
        gpu_s = gpu_ms * 1e-3
        cpu_args = (q, w["cell"], w["positions"], w["cutoff"], w["pbc"])
        cpu_fn(*cpu_args, types=types)
        ct = []
        for _ in range(3):
            t0 = time.perf_counter()
            res = cpu_fn(*cpu_args, types=types)
            ct.append(time.perf_counter() - t0)
        cpu_s = statistics.median(ct)
        # algorithmic bytes of the whole build: the outputs plus the inputs
        bq = sum({"i": 4, "j": 4, "D": 24, "d": 8, "S": 12}[c] for c in set(q))
        bin_ = 24 + (8 if pa is not None else 0) + (4 if types is not None else 0)
        alg = npairs * bq + nat * bin_
        row = {"natoms": nat, "npairs": npairs, "quantities": q,
               "gpu_ms": gpu_ms, "gpu_pairs_per_s": npairs / gpu_s,
               "stage_ms": {"count_phase": count_ms, "fill": fill_ms},
               "algorithmic_bytes": alg,
               "hbm_frac_whole_build": alg / gpu_s / 1e9 / peak,
               "hbm_frac_fill": alg / (fill_ms * 1e-3) / 1e9 / peak,
               "peak_gbs": peak, "peak_source": peak_kind,
               "cpu_ms": cpu_s * 1e3, "cpu_pairs_per_s": npairs / cpu_s,
               "cpu": {"kind": "reference" if have_ref else "port",
                       "cores": cores if have_ref else 1},
               "speedup": cpu_s / gpu_s}
        if len(grids) > 1:
            row["grids_ms"] = {g: v[0] for g, v in grid_rows.items()}
        if passes:
            row["pair_passes_ms"] = passes
        if check:
            # the bufs hold the last grid's build; every grid gives the same list
            row["parity"] = _same_device(q, [bufs[c] for c in q], res)
        del res
        if name.startswith("C5"):
            off = torch.empty(nat + 1, dtype=torch.int64, device=dev)
            ext.check(ext.lib.nbl_row_offsets(plan, ctypes.c_void_p(off.data_ptr()), sptr))
            gen = torch.Generator(device=dev).manual_seed(0)
            gD = torch.randn((npairs, 3), dtype=torch.float64, device=dev, generator=gen)
            gd = torch.randn(npairs, dtype=torch.float64, device=dev, generator=gen)
            gpos = torch.empty((nat, 3), dtype=torch.float64, device=dev)
            gcell = torch.empty(9, dtype=torch.float64, device=dev)
            a = BackwardArgs()
            a.npairs, a.nat = npairs, nat
            a.first, a.second = bufs["i"].data_ptr(), bufs["j"].data_ptr()
            a.shift, a.distvec = bufs["S"].data_ptr(), bufs["D"].data_ptr()
            a.absdist = bufs["d"].data_ptr()
            a.grad_distvec, a.grad_absdist = gD.data_ptr(), gd.data_ptr()
            a.row_offsets = off.data_ptr()
            a.pbc = pbc8.ctypes.data
            a.grad_positions, a.grad_cell = gpos.data_ptr(), gcell.data_ptr()
            bl = _lib()
            for det in (0, 1):
                a.deterministic = det
                # enqueued back to back (L2 flush between calls, outside the
                # events), so the events time the device work, not the host
                evs = []
                for k in range(reps + 3):
                    flush.zero_()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    ext.check(bl.nbl_backward(ctypes.byref(a), sptr))
                    e1.record(stream)
                    evs.append((e0, e1))
                torch.cuda.synchronize(dev)
                bms = [e0.elapsed_time(e1) for e0, e1 in evs[3:]]
                bt = statistics.median(bms) * 1e-3
                alg = npairs * 84 + nat * 48
                row["backward_deterministic" if det else "backward"] = {
                    "ms": bt * 1e3, "achieved_gbs": alg / bt / 1e9,
                    "frac": alg / bt / 1e9 / peak, "peak_gbs": peak,
                    "peak_source": peak_kind, "algorithmic_bytes": alg}
        if name.startswith("C5"):
            # CSR helpers on the device: row starts, then the triplets of pairs
            # shorter than 3.5 A (the first shell) -- against the reference's
            # own first_neighbours / triplet_list on the host (serial code)
            tcut = 3.5
            seed = torch.empty(nat + 1, dtype=torch.int32, device=dev)
            dt = bufs["d"]
            n3 = ctypes.c_int64()
            fms, tms = [], []
            for k in range(reps + 3):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e2 = torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize(dev)
                e0.record(stream)
                ext.check(ext.lib.nbl_first_neighbours(nat, npairs,
                                                       ctypes.c_void_p(bufs["i"].data_ptr()),
                                                       ctypes.c_void_p(seed.data_ptr()), sptr))
                e1.record(stream)
                ext.check(ext.lib.nbl_triplet_list(nat + 1, ctypes.c_void_p(seed.data_ptr()),
                                                   ctypes.c_void_p(dt.data_ptr()), tcut, None,
                                                   None, 0, ctypes.byref(n3), sptr))
                if k == 0:
                    tij = torch.empty(n3.value, dtype=torch.int32, device=dev)
                    tik = torch.empty(n3.value, dtype=torch.int32, device=dev)
                ext.check(ext.lib.nbl_triplet_list(nat + 1, ctypes.c_void_p(seed.data_ptr()),
                                                   ctypes.c_void_p(dt.data_ptr()), tcut,
                                                   ctypes.c_void_p(tij.data_ptr()),
                                                   ctypes.c_void_p(tik.data_ptr()), n3.value,
                                                   ctypes.byref(n3), sptr))
                e2.record(stream)
                e2.synchronize()
                if k >= 3:
                    fms.append(e0.elapsed_time(e1))
                    tms.append(e1.elapsed_time(e2))
            seed_h = seed.cpu().numpy()
            d_h = dt.cpu().numpy()
            ct = []
            for _ in range(3):
                t0 = time.perf_counter()
                if have_ref:
                    O.ref_first_neighbours(nat, bufs["i"].cpu().numpy())
                    O.ref_triplet_list(seed_h, d_h, tcut)
                else:
                    O.oracle_first_neighbours(nat, bufs["i"].cpu().numpy())
                    O.oracle_triplet_list(seed_h, d_h, tcut)
                ct.append(time.perf_counter() - t0)
            row["csr_helpers"] = {
                "first_neighbours_ms": statistics.median(fms),
                "triplet_list_ms": statistics.median(tms),
                "triplet_cutoff_A": tcut, "ntriplets": int(n3.value),
                "note": "triplet_list = count call + fill call (each synchronises once)",
                "cpu_ms": 1e3 * statistics.median(ct),
                "cpu": {"kind": "reference" if have_ref else "port", "cores": 1}}
        out[name] = row

    if wanted("verlet_C2"):
        _verlet_line(out, dev, flush, reps, stream, W)
    if wanted("LJ_droplet_1M"):
        _lj_line(out, dev, flush, reps, stream, sptr, plan, W, O, ext, have_ref, cpu_fn, cores)
    return out


def _verlet_line(out, dev, flush, reps, stream, W):
    """List reuse across steps (VerletList) on the dense bulk workload: the
    rebuild (cutoff + skin) against a refresh after a small displacement,
    both through update() (its host synchronisations included)."""
    import torch
    from matscipy_neighbours.verlet import VerletList
    wv = W.fcc_bulk(seed=0)
    posv = torch.from_numpy(wv["positions"]).to(dev)
    skin = 0.5
    vl = VerletList(cutoff=wv["cutoff"], skin=skin, cell=wv["cell"], pbc=wv["pbc"])
    gen = torch.Generator(device=dev).manual_seed(0)
    kick = 0.01 * torch.randn(posv.shape, dtype=torch.float64, device=dev, generator=gen)
    bms, rms = [], []
    for k in range(reps + 3):
        vl._stored = None  # force a rebuild
        flush.zero_()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e2 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = vl.update(posv)
        e1.record(stream)
        del res
        flush.zero_()
        e1b = torch.cuda.Event(enable_timing=True)
        e1b.record(stream)
        res = vl.update(posv + kick)
        e2.record(stream)
        e2.synchronize()
        del res
        if k >= 3:
            bms.append(e0.elapsed_time(e1))
            rms.append(e1b.elapsed_time(e2))
    out["verlet_C2"] = {"natoms": int(posv.shape[0]), "cutoff": wv["cutoff"], "skin": skin,
                        "stored_pairs": int(vl._stored[0].shape[0]),
                        "rebuild_ms": statistics.median(bms),
                        "refresh_ms": statistics.median(rms),
                        "refreshes": vl.refreshes, "builds": vl.builds}
    del vl, posv, kick


def _lj_line(out, dev, flush, reps, stream, sptr, plan, W, O, ext, have_ref, cpu_fn, cores):
    """The fused consumer on the reference's molecular-dynamics benchmark
    system: LJ forces and energy of a 1,000,000-atom FCC droplet (reduced
    units, lattice 1.6, cutoff 2.5, open box) with no pair list written
    (nbl_lj_forces), against the reference's CPU core building the pair list
    (all host threads) plus float64 numpy force sums."""
    import ctypes

    import numpy as np
    import torch
    w = W.lj_droplet()
    nat = w["positions"].shape[0]
    cell = np.ascontiguousarray(w["cell"], dtype=float)
    inv = np.ascontiguousarray(np.linalg.inv(cell.T))
    pbc8 = np.zeros(3, dtype=np.uint8)
    pos = torch.from_numpy(w["positions"]).to(dev)
    req = ext.make_request(ext.QUANTITY_FIRST, np.zeros(3), cell, inv, pbc8, nat,
                           ctypes.c_void_p(pos.data_ptr()), True, w["cutoff"], None, None,
                           0, None, dev.index)
    forces = torch.empty((nat, 3), dtype=torch.float64, device=dev)
    energy = torch.empty((), dtype=torch.float64, device=dev)
    evs = []
    for k in range(reps + 3):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ext.check(ext.lib.nbl_lj_forces(plan, ctypes.byref(req), 1.0, 1.0,
                                        ctypes.c_void_p(forces.data_ptr()),
                                        ctypes.c_void_p(energy.data_ptr()), sptr))
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize(dev)
    ext.check(ext.lib.nbl_check(plan, sptr))
    gms = statistics.median([e0.elapsed_time(e1) for e0, e1 in evs[3:]])
    n = ctypes.c_int64()
    ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), sptr, ctypes.byref(n)))

    def cpu_lj():
        i, D, d = cpu_fn("iDd", w["cell"], w["positions"], w["cutoff"], w["pbc"])
        s6 = (1.0 / (d * d)) ** 3
        coef = -24.0 * s6 * (2.0 * s6 - 1.0) / (d * d)
        f = np.stack([np.bincount(i, weights=coef * D[:, k], minlength=nat)
                      for k in range(3)], axis=1)
        return 0.5 * float(np.sum(4.0 * (s6 * s6 - s6))), f

    t0 = time.perf_counter()
    e_cpu, f_cpu = cpu_lj()
    cpu_s = time.perf_counter() - t0
    out["LJ_droplet_1M"] = {
        "natoms": nat, "npairs": int(n.value), "cutoff": w["cutoff"],
        "gpu_ms": gms, "gpu_pairs_per_s": n.value / (gms * 1e-3),
        "what": "nbl_lj_forces: bin + count + force pass, no pairs written",
        "energy_rel_diff_vs_cpu": abs(float(energy.item()) - e_cpu) / abs(e_cpu),
        "forces_max_abs_diff_vs_cpu": float(np.abs(forces.cpu().numpy() - f_cpu).max()),
        "cpu_ms": cpu_s * 1e3,
        "cpu": {"kind": ("reference" if have_ref else "port") + " pair list + numpy forces",
                "cores": cores if have_ref else 1},
        "speedup": cpu_s / (gms * 1e-3)}


def _cpu_fn(O, cores):
    """The reference's own core (oracle/_ref, OpenMP, `cores` threads) when it
    was built, else the C restatement (one thread)."""
    if O.ref_available():
        O.ref_set_threads(cores)
        return "reference", cores, O.ref_neighbour_list
    return "port", 1, O.oracle_neighbour_list


def per_call_latency(dev, sizes=(100, 1000), calls=60):
    """Host-clock latency of one whole call on small systems (random gas,
    0.08 atoms/A^3, rc 4 A, all five outputs): through the C-ABI with device
    positions and device outputs (nbl_count + nbl_fill, then a stream
    synchronisation), and through the public neighbour_list with numpy in and
    numpy out.  Median over `calls` calls after 10 warm-up calls."""
    import ctypes

    import numpy as np
    import torch

    import matscipy_neighbours as m
    from matscipy_neighbours import _matscipy_neighbours as ext
    rng = np.random.default_rng(0)
    out = {}
    for nat in sizes:
        L = (nat / 0.08) ** (1.0 / 3.0)
        pos = np.ascontiguousarray(rng.uniform(0.0, L, size=(nat, 3)))
        cell = L * np.eye(3)
        inv = np.ascontiguousarray(np.linalg.inv(cell.T))
        pbc8 = np.ones(3, dtype=np.uint8)
        origin = np.zeros(3)
        pos_d = torch.from_numpy(pos).to(dev)
        stream = torch.cuda.current_stream(dev)
        sp = ctypes.c_void_p(stream.cuda_stream)
        plan = ext.plan_for(dev.index)
        req = ext.make_request(31, origin, cell, inv, pbc8, nat, ctypes.c_void_p(pos_d.data_ptr()),
                               True, 4.0, None, None, 0, None, dev.index)
        n = ctypes.c_int64()
        ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), sp, ctypes.byref(n)))
        bufs = {c: torch.empty((n.value,) + ext._SHAPES[c][0],
                               dtype=torch.int32 if ext._SHAPES[c][1] == np.int32
                               else torch.float64, device=dev) for c in "ijdDS"}
        o = ext._outputs_struct(bufs, lambda t: t.data_ptr())

        def abi():
            ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), sp, ctypes.byref(n)))
            ext.check(ext.lib.nbl_fill(plan, ctypes.byref(o), sp))
            stream.synchronize()

        def api():
            m.neighbour_list("ijdDS", positions=pos, cell=cell, pbc=True, cutoff=4.0)

        res = {"npairs": int(n.value)}
        for name, f in (("c_abi_device_us", abi), ("python_api_host_us", api)):
            ts = []
            for k in range(calls + 10):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                f()
                if k >= 10:
                    ts.append(time.perf_counter() - t0)
            res[name] = round(1e6 * statistics.median(ts), 1)
        out[str(nat)] = res
    return out


def workload_config(nat, reps, npairs, world):
    """The `config` object of both arms' JSON lines (identical on purpose)."""
    return dict(WORKLOAD, natoms=nat, reps=reps, npairs_per_step=npairs,
                parallelism=f"replicas{world}",
                l2="working set larger than L2 (2.5 GB of pairs written per step); "
                   "the GPU arm also flushes L2 (256 MiB write) between steps")


def cpu_baseline(steps=2, want=None):
    """The reference's CPU core on the same workload (rank 0, N = 1), every
    host thread, plus a one-thread row on a bounded sample (32^3 FCC cells,
    1/8 of the workload) for context.  With `want` (a callable taking the
    core's full "ijdDS" result) the last full result is handed over before it
    is freed, for the parity check."""
    O = _oracle()
    W = _workloads()
    w = W.fcc_bulk(seed=0)
    cores = len(os.sched_getaffinity(0))
    kind, cores, fn = _cpu_fn(O, cores)
    fn("ijdDS", w["cell"], w["positions"], w["cutoff"], w["pbc"])  # warm-up
    times, npairs = [], 0
    for k in range(steps):
        t0 = time.perf_counter()
        res = fn("ijdDS", w["cell"], w["positions"], w["cutoff"], w["pbc"])
        times.append(time.perf_counter() - t0)
        npairs = len(res[0])
        if want is not None and k == steps - 1:
            want(res)
        del res
    med = statistics.median(times)
    out = {"value": npairs / med, "unit": UNIT, "cores": cores, "kind": kind,
           "sample": f"full workload ({npairs} pairs), median of {steps} calls",
           "seconds_per_call": med}
    if kind == "reference":
        ws = W.fcc_bulk(seed=0, reps=32)
        O.ref_set_threads(1)
        fn("ijdDS", ws["cell"], ws["positions"], ws["cutoff"], ws["pbc"])
        t1 = []
        for _ in range(3):
            t0 = time.perf_counter()
            n1 = len(fn("ijdDS", ws["cell"], ws["positions"], ws["cutoff"], ws["pbc"])[0])
            t1.append(time.perf_counter() - t0)
        O.ref_set_threads(cores)
        m1 = statistics.median(t1)
        out["one_thread"] = {"value": n1 / m1, "unit": UNIT, "cores": 1, "kind": kind,
                             "sample": f"32^3 FCC cells (131072 atoms, {n1} pairs), "
                                       f"median of 3 calls",
                             "seconds_per_call": m1}
    return out


def reference_gpu_bench(dev, w, pos_d, outs, npairs, reps=9):
    """The reference's own CUDA backend (oracle/_ref/libref_gpu.so: its
    neighbour_list_gpu_device compiled for sm_100a from its sources) on the
    same device-resident workload, as a secondary comparator: the device time
    of its call (its own allocations, copies and synchronisations included),
    median of `reps` after one warm-up; and its pairs against the engine's,
    canonically ordered by (i, j) since its row order is not the reference
    CPU's: the same (i, j, S) and the largest |D|, |d| differences."""
    import torch
    O = _oracle()
    if not O.refgpu_available():
        return {"unavailable": "oracle/_ref/libref_gpu.so not built (reference sources "
                               "absent when build() ran)"}
    nat = pos_d.shape[0]
    # the reference allocates its 2.5 GB of outputs with cudaMalloc on every
    # call: give it the memory torch's caching allocator holds
    torch.cuda.synchronize(dev)
    torch.cuda.empty_cache()
    ref = {"i": torch.empty(npairs, dtype=torch.int32, device=dev),
           "j": torch.empty(npairs, dtype=torch.int32, device=dev),
           "D": torch.empty((npairs, 3), dtype=torch.float64, device=dev),
           "d": torch.empty(npairs, dtype=torch.float64, device=dev),
           "S": torch.empty((npairs, 3), dtype=torch.int32, device=dev)}
    torch.cuda.synchronize(dev)
    n, _ = O.refgpu_neighbour_list("ijDdS", w["cell"], pos_d.data_ptr(), nat, w["cutoff"],
                                   w["pbc"], outputs=[ref[q].data_ptr() for q in "ijDdS"],
                                   capacity=npairs)
    ms = []
    for _ in range(reps):
        _, t = O.refgpu_neighbour_list("ijdDS", w["cell"], pos_d.data_ptr(), nat, w["cutoff"],
                                       w["pbc"])
        ms.append(t)
    out = {"what": "reference neighbour_list_gpu_device (its CUDA backend, sm_100a build)",
           "npairs": n, "ms_per_build": statistics.median(ms), "ms_min": min(ms),
           "ms_samples": ms,
           "value": n / (statistics.median(ms) * 1e-3), "unit": UNIT}
    if n == npairs:
        def canon(o):
            key = o["i"].to(torch.int64) * nat + o["j"].to(torch.int64)
            order = torch.sort(key, stable=True).indices
            return key[order], o["S"][order], o["D"][order], o["d"][order]
        ka, sa, da, aa = canon(ref)
        kb, sb, db, ab = canon(outs)
        out["same_ij_S"] = bool(torch.equal(ka, kb) and torch.equal(sa, sb))
        out["max_abs_diff_D"] = float((da - db).abs().max()) if npairs else 0.0
        out["max_abs_diff_d"] = float((aa - ab).abs().max()) if npairs else 0.0
        del ka, sa, da, aa, kb, sb, db, ab
    else:
        out["same_ij_S"] = False
    del ref
    torch.cuda.empty_cache()
    return out


def run_reference(args, rank):
    """The reference's own CPU core (oracle/_ref: its neighbour_list.cc and
    cell_list.cc compiled from source, OpenMP) on every host thread, on the
    full benchmark workload: each step is one complete "ijdDS" build of the
    1,048,576-atom sheared FCC bulk.  Nothing of the engine is loaded in this
    process (the generators come from their own file).  Under torchrun only
    rank 0 runs; the other ranks exit without work."""
    if rank != 0:
        return
    O = _oracle()
    W = _workloads()
    w = W.fcc_bulk(seed=0, reps=args.reps)
    nat = w["positions"].shape[0]
    cores = len(os.sched_getaffinity(0))
    kind, cores, fn = _cpu_fn(O, cores)
    for _ in range(args.warmup):
        fn("ijdDS", w["cell"], w["positions"], w["cutoff"], w["pbc"])
    times, npairs = [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        npairs = len(fn("ijdDS", w["cell"], w["positions"], w["cutoff"], w["pbc"])[0])
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = npairs * args.steps / total
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(nat, args.reps, npairs, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"the full workload every step ({nat} atoms, "
                                   f"{npairs} pairs), host wall clock per call"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own CUDA backend")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the bit-for-bit comparisons with the CPU checker")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the C1/C3/C5 lines (and the backward timing)")
    ap.add_argument("--only-configs", default=None,
                    help="comma-separated config lines to run alone (e.g. C5_diff_lattice, "
                         "LJ_droplet_1M, verlet_C2); prints them and nothing else")
    ap.add_argument("--thread-per-atom", default="auto", choices=["auto", "on", "off"],
                    help="pair passes of the C1/C3/C5/dilute-gas lines: the default "
                         "choice, one thread per atom, or one warp per work item")
    ap.add_argument("--reps", type=int, default=64,
                    help="FCC unit cells per edge (64 = the benchmark size; smaller "
                         "values make the small cases used for profiling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import ctypes

    import numpy as np
    import torch

    import matscipy_neighbours as m
    from matscipy_neighbours import _matscipy_neighbours as ext
    W = _workloads()

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.only_configs:
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
        only = set(x.strip() for x in args.only_configs.split(",") if x.strip())
        tpa = {"auto": 0, "on": 1, "off": -1}[args.thread_per_atom]
        print(json.dumps({"configs": configs_bench(dev, flush, only=only,
                                                   thread_per_atom=tpa)}), flush=True)
        return
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    w = W.fcc_bulk(seed=rank, reps=args.reps)
    nat = w["positions"].shape[0]
    cell = np.ascontiguousarray(w["cell"])
    inv = np.ascontiguousarray(np.linalg.inv(cell.T))
    origin = np.zeros(3)
    pbc8 = np.ones(3, dtype=np.uint8)
    pos_d = torch.from_numpy(w["positions"]).to(dev)
    stream = torch.cuda.Stream(dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    plan = ext.plan_for(local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def request(precision):
        prev = ext.set_options(precision=precision, grid="auto")
        r = ext.make_request(31, origin, cell, inv, pbc8, nat,
                             ctypes.c_void_p(pos_d.data_ptr()), True, w["cutoff"], None,
                             None, 0, None, local)
        ext.set_options(**{"precision": prev["precision"], "grid": prev["grid"]})
        return r

    npairs_c = ctypes.c_int64()
    req = request("fp32")
    with torch.cuda.stream(stream):
        ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), sptr, ctypes.byref(npairs_c)))
    npairs = int(npairs_c.value)
    outs = {"i": torch.empty(npairs, dtype=torch.int32, device=dev),
            "j": torch.empty(npairs, dtype=torch.int32, device=dev),
            "D": torch.empty((npairs, 3), dtype=torch.float64, device=dev),
            "d": torch.empty(npairs, dtype=torch.float64, device=dev),
            "S": torch.empty((npairs, 3), dtype=torch.int32, device=dev)}
    ostruct = ext._outputs_struct(outs, lambda t: t.data_ptr())

    def timed_steps(req, k, record=True):
        """k full builds; returns (per-step ms, per-fill ms)."""
        step_ms, fill_ms = [], []
        for _ in range(k):
            flush.zero_()
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e2 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ext.check(ext.lib.nbl_count(plan, ctypes.byref(req), sptr,
                                        ctypes.byref(npairs_c)))
            e1.record(stream)
            ext.check(ext.lib.nbl_fill(plan, ctypes.byref(ostruct), sptr))
            e2.record(stream)
            e2.synchronize()
            step_ms.append(e0.elapsed_time(e2))
            fill_ms.append(e1.elapsed_time(e2))
        return step_ms, fill_ms

    # --- FP32-filter path (the headline), then plain FP64 for comparison ----
    timed_steps(req, args.warmup)
    ext.check(ext.lib.nbl_check(plan, sptr))
    clocks = ClockSampler(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    ext.lib.nbl_launch_count(1)
    step_ms, fill_ms = timed_steps(req, args.steps)
    launches = int(ext.lib.nbl_launch_count(1))
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    clk = clocks.stop()
    ext.check(ext.lib.nbl_check(plan, sptr))

    step64 = fill64 = None
    if not args.no_fp64:
        req64 = request("fp64")
        timed_steps(req64, 2)
        step64, fill64 = timed_steps(req64, max(3, min(args.steps, 20)))

    total_ms = sum(step_ms)
    pairs_job = npairs * args.steps
    if dist is not None:
        t = torch.tensor([total_ms, float(pairs_job)], dtype=torch.float64, device=dev)
        tmax = t.clone()
        dist.all_reduce(tmax[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        total_ms, pairs_job = float(tmax[0]), float(t[1])
    value = pairs_job / (total_ms * 1e-3)

    # --- end to end through the public API with host buffers ----------------
    e2e_value = None
    e2e_times = []
    if not args.no_e2e:
        host_pos = ext.host_empty((nat, 3), np.float64)
        host_pos[...] = w["positions"]
        e2e_steps = min(args.steps, 10)
        for k in range(args.warmup + e2e_steps):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            res = m.neighbour_list("ijdDS", positions=host_pos, cell=cell, pbc=w["pbc"],
                                   cutoff=w["cutoff"])
            t1 = time.perf_counter()
            if k >= args.warmup:
                e2e_times.append(t1 - t0)
            del res
        e2e_total = sum(e2e_times)
        e2e_pairs = npairs * len(e2e_times)
        if dist is not None:
            t = torch.tensor([e2e_total, float(e2e_pairs)], dtype=torch.float64,
                             device=dev)
            tmax = t.clone()
            dist.all_reduce(tmax[:1], op=dist.ReduceOp.MAX)
            dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
            e2e_total, e2e_pairs = float(tmax[0]), float(t[1])
        e2e_value = e2e_pairs / e2e_total

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    peak, peak_kind, peaks = _peaks()
    fill_avg_s = statistics.mean(fill_ms) * 1e-3
    alg_bytes = npairs * BYTES_PER_PAIR + nat * BYTES_PER_ATOM_IN
    achieved = alg_bytes / fill_avg_s / 1e9
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(nat, args.reps, npairs, world),
        "precision": "fp32 filter + fp64 guard-band recheck",
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": _traffic_per_launch(npairs, nat),
                     "kernel": "k_fill (fill pass)",
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "fill_ms": statistics.mean(fill_ms)},
        "e2e": ({"value": e2e_value, "unit": UNIT,
                 "h2d_bytes_per_step": nat * 3 * 8,
                 "d2h_bytes_per_step": npairs * BYTES_PER_PAIR,
                 "ms_per_step": 1e3 * statistics.mean(e2e_times)}
                if e2e_value is not None else None),
        "gpu_launches": launches,
        "clocks": clk,
        "fp64_plain": ({"value": npairs / (statistics.mean(step64) * 1e-3),
                        "ms_per_step": statistics.mean(step64),
                        "fill_ms": statistics.mean(fill64)} if step64 else None),
        "stage_ms": {"count_phase": statistics.mean(a - b for a, b in zip(step_ms, fill_ms)),
                     "fill": statistics.mean(fill_ms)},
    }
    parity = {}
    if not args.no_batched:
        out["batched"] = batched_bench(min(args.steps, 20), args.warmup, dev, rank,
                                       check=world == 1 and not args.no_parity)
        if "parity" in out["batched"]:
            parity["C4"] = out["batched"]["parity"]
    if world == 1 and not args.no_configs:
        out["configs"] = configs_bench(dev, flush, check=not args.no_parity,
                                       thread_per_atom={"auto": 0, "on": 1,
                                                        "off": -1}[args.thread_per_atom])
        for name, key in (("C1_plain_small", "C1"), ("C3_sparse_slab", "C3"),
                          ("C5_diff_lattice", "C5"), ("gas_dilute", "gas_dilute")):
            if "parity" in out["configs"].get(name, {}):
                parity[key] = out["configs"][name]["parity"]
    if world == 1 and not args.no_configs:
        out["per_call_latency"] = per_call_latency(dev)
    if world == 1 and not args.no_cpu_baseline and args.reps == 64:
        want = None
        if not args.no_parity:
            # the headline build once more (FP32 filter), outside any timing,
            # compared with the reference core's last full result
            timed_steps(req, 1)
            ext.check(ext.lib.nbl_check(plan, sptr))

            def want(res):
                parity["C2"] = _same_device("ijdDS", [outs[q] for q in "ijdDS"], res)
        out["cpu_baseline"] = cpu_baseline(want=want)
    if world == 1 and not args.no_reference_gpu and args.reps == 64:
        timed_steps(req, 1)
        ext.check(ext.lib.nbl_check(plan, sptr))
        rg = reference_gpu_bench(dev, w, pos_d, outs, npairs)
        if "ms_per_build" in rg:
            rg["engine_speedup"] = rg["ms_per_build"] / (total_ms / args.steps)
        out["reference_gpu"] = rg
    if parity:
        out["parity"] = parity
        out["parity_checker"] = ("oracle/_ref (the reference's own CPU core, compiled from its "
                                 "sources)" if _oracle().ref_available()
                                 else "oracle (C restatement of the reference CPU path)")
    print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
