"""Continuous-batching request loop for projector jobs on one GPU.

A stream of jobs (forward projection or backprojection, 2D fan or 3D cone, any
geometry, FP32/BF16/FP16 storage) arrives over time.  The server

* admits jobs while execution slots and HBM are free (memory admission: a
  class's buffer set and the batch's result copies must fit the free device
  memory above a reserve; idle buffer sets of other classes are evicted,
  oldest first, to make room);
* groups ready jobs of one *class* (same op, geometry, dtype) into one batched
  launch -- the C ABI runs a whole batch in one launch with shared geometry;
* keeps per-class device-resident buffers, geometry and workspaces (two
  buffer sets per class, so two batches of one class can be in flight), and
  replays a CUDA graph captured per (class, batch size, buffer set) once
  warmed up; results stay on the device;
* spreads batches over several CUDA streams so they overlap on the device,
  and retires each batch when its completion event has fired, admitting
  newly arrived jobs as soon as slots and memory free up;
* runs short job classes on high-priority streams: a large job's kernel
  fills every SM, and without priorities a short job launched beside it
  waits until the large kernel's blocks have all started; with them the
  block scheduler starts the short job's blocks first.

Latency of a job = completion seen by the host - arrival.  ``run_trace``
returns per-job latencies, p50/p99 and aggregate GUPS (updates: voxels x views
for every job, forward and back alike).

Each batch element is computed exactly as it would be alone (batching only
widens the grid), so results are bitwise the same alone and in the mix.
"""
from __future__ import annotations

import collections
import dataclasses
import math
import time
import zlib
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

from . import geometry as _geometry
from . import phantoms as _phantoms


# ----------------------------------------------------------------- job model


@dataclasses.dataclass(frozen=True)
class JobClass:
    """Everything that must match for two jobs to share one launch."""
    op: str            # "fan_fwd", "fan_bp", "cone_fwd", "cone_bp"
    geometry: str      # key into the server's geometry table
    dtype: str         # "fp32", "bf16", "fp16"


@dataclasses.dataclass
class Job:
    id: int
    cls: JobClass
    data: object              # host (pinned) or device tensor: the op input without batch dim
    arrival: float            # seconds, trace time
    updates: int = 0          # voxels x views
    admit: float = math.nan
    done: float = math.nan
    result: object = None

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclasses.dataclass
class ServeStats:
    latencies_ms: np.ndarray
    p50_ms: float
    p99_ms: float
    gups: float
    wall_s: float
    batches: int
    mean_batch: float
    graph_replays: int
    per_class: dict = dataclasses.field(default_factory=dict)  # "geometry/op" -> {n, p50_ms, p99_ms}

    def as_dict(self):
        return {"p50_ms": self.p50_ms, "p99_ms": self.p99_ms, "gups": self.gups, "wall_s": self.wall_s,
                "batches": self.batches, "mean_batch": self.mean_batch, "graph_replays": self.graph_replays,
                "jobs": int(self.latencies_ms.size), "per_class": self.per_class}


def per_class_latency(jobs) -> dict:
    """p50 / p99 latency (ms) per geometry and op (dtypes pooled)."""
    groups = collections.defaultdict(list)
    for j in jobs:
        groups["%s/%s" % (j.cls.geometry, j.cls.op)].append((j.done - j.arrival) * 1e3)
    return {k: {"n": len(v), "p50_ms": percentile(v, 50), "p99_ms": percentile(v, 99)}
            for k, v in sorted(groups.items())}


def percentile(values, q):
    v = np.sort(np.asarray(values, dtype=np.float64))
    if v.size == 0:
        return math.nan
    return float(np.percentile(v, q))


# ------------------------------------------------------------ geometry table


@dataclasses.dataclass
class GeometryEntry:
    kind: str                       # "fan" or "cone"
    geo: object                     # geometry.FanBeam2D / geometry.ConeBeam3D
    volume_shape: Tuple[int, ...]
    sinogram_shape: Tuple[int, ...]

    @property
    def updates(self) -> int:
        return int(np.prod(self.volume_shape)) * int(self.sinogram_shape[0])


def standard_geometries() -> Dict[str, GeometryEntry]:
    """The serving mix's geometries: 2D fan 512^2 (360 views, 1024 px at
    0.5 mm, SID 750 / SDD 1200), cone 128^3 (180 views, 256^2 at 1.5 mm, SID
    600 / SDD 1000, 1 mm voxels) and cone 256^3 (360 views, 512^2 at 1 mm,
    0.5 mm voxels, SID 750 / SDD 1200)."""
    fan = _geometry.FanBeam2D((512, 512), (0.5, 0.5), 1024, 0.5, 360, 750.0, 1200.0)
    c128 = _geometry.ConeBeam3D((128, 128, 128), (1.0, 1.0, 1.0), (256, 256), (1.5, 1.5), 180, 600.0, 1000.0)
    c256 = _geometry.ConeBeam3D((256, 256, 256), (0.5, 0.5, 0.5), (512, 512), (1.0, 1.0), 360, 750.0, 1200.0)
    return {
        "fan512": GeometryEntry("fan", fan, fan.volume_shape, fan.detector_shape),
        "cone128": GeometryEntry("cone", c128, c128.volume_shape, c128.detector_shape),
        "cone256": GeometryEntry("cone", c256, c256.volume_shape, c256.detector_shape),
    }


def poisson_trace(n_jobs: int, rate_hz: float, seed: int, mix=None) -> List[Tuple[float, JobClass]]:
    """Seeded arrival trace: exponential inter-arrival times at rate_hz; each
    job draws its geometry from mix (name -> probability), forward/back 50/50
    and FP32/BF16 50/50."""
    mix = mix or {"fan512": 0.6, "cone128": 0.3, "cone256": 0.1}
    rng = np.random.Generator(np.random.PCG64(seed))
    names = list(mix)
    probs = np.array([mix[n] for n in names], dtype=np.float64)
    probs /= probs.sum()
    t = 0.0
    out = []
    for _ in range(n_jobs):
        t += rng.exponential(1.0 / rate_hz)
        name = names[int(rng.choice(len(names), p=probs))]
        kind = "fan" if name.startswith("fan") else "cone"
        op = kind + ("_fwd" if rng.random() < 0.5 else "_bp")
        dtype = "fp32" if rng.random() < 0.5 else "bf16"
        out.append((t, JobClass(op, name, dtype)))
    return out


# ------------------------------------------------------------- execution


class Executor:
    """Runs batches of one job class on the GPU through the C ABI.

    Holds up to n_sets buffer sets (input, output, workspace sized for
    max_batch jobs; a batch of b jobs uses the first b); a set serves one
    in-flight batch at a time.  After two eager runs of a (batch size, set)
    the launch sequence is captured as a CUDA graph and replayed."""

    def __init__(self, cls: JobClass, entry: GeometryEntry, device, max_batch: int, use_graphs: bool = True,
                 n_sets: int = 2):
        import torch

        from . import _capi, ops
        self.torch, self._capi, self.ops = torch, _capi, ops
        self.cls = cls
        self.entry = entry
        self.device = device
        self.max_batch = max_batch
        self.dtype = {"fp32": torch.float32, "bf16": torch.bfloat16, "fp16": torch.float16}[cls.dtype]
        self.fwd = cls.op.endswith("_fwd")
        self.in_shape = entry.volume_shape if self.fwd else entry.sinogram_shape
        self.out_shape = entry.sinogram_shape if self.fwd else entry.volume_shape
        # results of backprojections are volumes: keep them FP32
        self.out_dtype = self.dtype if self.fwd else torch.float32
        self.use_graphs = use_graphs
        self.n_sets = n_sets
        self.busy = [False] * n_sets
        self.last_use = [0.0] * n_sets
        self._sets = {}      # set -> (inp, out, ws)
        self._graphs = {}    # (batch, set) -> torch.cuda.CUDAGraph
        self._runs = {}      # (batch, set) -> eager runs so far
        self._cap = None     # side stream for graph captures
        self.graph_replays = 0
        g = entry.geo
        if entry.kind == "fan":
            self.geo = ops.Geometry2D(1, device, g.volume_origin, g.detector_origin, g.volume_spacing,
                                      g.detector_spacing, g.ray_vectors, g.detector_shape[0], g.sid, g.sdd)
        else:
            self.geo = ops.GeometryCone(1, device, *g.args(), g.detector_shape[0])

    def _elem(self, dtype) -> int:
        return self.torch.tensor([], dtype=dtype).element_size()

    def result_bytes(self, batch: int) -> int:
        return batch * int(np.prod(self.out_shape)) * self._elem(self.out_dtype)

    def set_bytes(self) -> int:
        b = self.max_batch
        return b * (int(np.prod(self.in_shape)) * self._elem(self.dtype) +
                    int(np.prod(self.out_shape)) * self._elem(self.out_dtype)) + self._ws_bytes(b)

    def _ws_bytes(self, batch: int) -> int:
        code = self.ops.storage_code(self.dtype)
        if self.entry.kind == "fan":
            if not self.fwd:
                return 0
            return self._capi.workspace_size("pyronn_projection2d", batch, *self.in_shape, code)
        name = "pyronn_cone_projection3d" if self.fwd else "pyronn_cone_backprojection3d"
        return self._capi.workspace_size(name, batch, *self.in_shape, *self.out_shape, code, 0, 1)

    def allocated(self, bset: int) -> bool:
        return bset in self._sets

    def free_set(self) -> Optional[int]:
        for i, b in enumerate(self.busy):
            if not b:
                return i
        return None

    def allocate(self, bset: int):
        if bset not in self._sets:
            t = self.torch
            b = self.max_batch
            inp = t.zeros((b,) + tuple(self.in_shape), dtype=self.dtype, device=self.device)
            out = t.empty((b,) + tuple(self.out_shape), dtype=self.out_dtype, device=self.device)
            ws = t.empty(max(self._ws_bytes(b), 1), dtype=t.uint8, device=self.device)
            self._sets[bset] = (inp, out, ws)
        return self._sets[bset]

    def evict(self, bset: int) -> int:
        """Drops an idle set's buffers and graphs; returns the bytes freed."""
        if bset not in self._sets or self.busy[bset]:
            return 0
        for key in [k for k in self._graphs if k[1] == bset]:
            del self._graphs[key]
        for key in [k for k in self._runs if k[1] == bset]:
            del self._runs[key]
        del self._sets[bset]
        return self.set_bytes()

    def _launch(self, batch: int, bset: int, stream_handle: int):
        inp, out, ws = self._sets[bset]
        code_in = self.ops.storage_code(self.dtype)
        code_out = self.ops.storage_code(self.out_dtype)
        if self.entry.kind == "fan":
            vol_y, vol_x = self.entry.volume_shape
            n_proj, det_w = self.entry.sinogram_shape
            if self.fwd:
                self._capi.call("pyronn_fan_projection2d", inp.data_ptr(), out.data_ptr(), code_in, code_out, batch,
                                vol_y, vol_x, n_proj, det_w, *self.geo.pointers(), 1, ws.data_ptr(), ws.numel(),
                                stream_handle)
            else:
                self._capi.call("pyronn_fan_backprojection2d", inp.data_ptr(), out.data_ptr(), code_in, code_out,
                                batch, n_proj, det_w, vol_y, vol_x, *self.geo.pointers(), 1, stream_handle)
        else:
            vz, vy, vx = self.entry.volume_shape
            n_proj, dh, dw = self.entry.sinogram_shape
            if self.fwd:
                self._capi.call("pyronn_cone_projection3d", inp.data_ptr(), out.data_ptr(), code_in, code_out, 0,
                                batch, vz, vy, vx, n_proj, dh, dw, *self.geo.pointers(), 1, ws.data_ptr(),
                                ws.numel(), stream_handle)
            else:
                self._capi.call("pyronn_cone_backprojection3d", inp.data_ptr(), out.data_ptr(), code_in, code_out, 0,
                                batch, n_proj, dh, dw, vz, vy, vx, *self.geo.pointers(), 1, ws.data_ptr(),
                                ws.numel(), stream_handle)
                # the batch's device error flag into the device's error word
                # (on the batch's stream; captured with the launch)
                self.ops.note_workspace_error(ws, self.device)

    def run(self, batch: int, bset: int, stream) -> None:
        """Enqueues the batch's kernels on stream (eager for the first runs,
        then as a CUDA graph replay)."""
        t = self.torch
        key = (batch, bset)
        if self.use_graphs and key in self._graphs:
            with t.cuda.stream(stream):
                self._graphs[key].replay()
            self.graph_replays += 1
            return
        with t.cuda.stream(stream):
            self._launch(batch, bset, stream.cuda_stream)
        n = self._runs.get(key, 0) + 1
        self._runs[key] = n
        if self.use_graphs and n >= 2:
            # capture after a warm-up run (lazy one-time set-up happens
            # eagerly), on a side stream ordered after this batch.  The launch
            # sequence allocates nothing, so the capture needs none of the
            # device-wide synchronisation, garbage collection and cache
            # flush that torch.cuda.graph() performs on entry -- in a serving
            # loop those stall every stream for the length of the longest
            # batch in flight.
            g = t.cuda.CUDAGraph()
            cap = self._capture_stream()
            cap.wait_stream(stream)
            with t.cuda.stream(cap):
                g.capture_begin()
                try:
                    self._launch(batch, bset, cap.cuda_stream)
                finally:
                    g.capture_end()
            stream.wait_stream(cap)
            self._graphs[key] = g

    def _capture_stream(self):
        if self._cap is None:
            self._cap = self.torch.cuda.Stream(self.device)
        return self._cap

    def prepare(self, batch: int, stream) -> None:
        """Allocates every buffer set and records the graphs of a batch size
        (two eager runs per set; results are not meaningful)."""
        for bset in range(self.n_sets):
            self.allocate(bset)
            while self.use_graphs and (batch, bset) not in self._graphs:
                self.run(batch, bset, stream)


class ProjectorServer:
    """Continuous batching over a fixed set of geometries (see module doc)."""

    def __init__(self, geometries: Dict[str, GeometryEntry], device=None, max_inflight: int = 8,
                 max_batch: int = 8, n_streams: int = 4, hbm_reserve: int = 4 << 30, use_graphs: bool = True,
                 keep_results: bool = True, clock: Callable[[], float] = time.perf_counter):
        import torch
        self.torch = torch
        self.device = torch.device(device or "cuda")
        self.geometries = geometries
        self.max_inflight = max_inflight
        self.max_batch = max_batch
        self.streams = [torch.cuda.Stream(self.device) for _ in range(n_streams)]
        # high-priority streams for short classes (lower number = higher priority)
        _, hi = torch.cuda.Stream.priority_range() if hasattr(torch.cuda.Stream, "priority_range") else (0, -1)
        self.fast_streams = [torch.cuda.Stream(self.device, priority=hi) for _ in range(max(1, n_streams // 2))]
        largest = max((e.updates for e in geometries.values()), default=1)
        self.short_updates = largest // 8  # classes at most this large are short
        self.hbm_reserve = hbm_reserve  # HBM always left free
        self.use_graphs = use_graphs
        self.keep_results = keep_results
        self.evictions = 0
        self._budget = 0  # bytes known free above the reserve (refreshed from the device when short)
        self.clock = clock
        self.executors: Dict[JobClass, Executor] = {}
        self.batches = 0
        self.batch_sizes = []

    def register_geometry(self, name: str, descriptor: dict) -> GeometryEntry:
        """Adds a geometry from its wire descriptor (wire.geometry_descriptor
        or wire.circular_descriptor) under name; requests refer to it."""
        from . import wire
        if name in self.geometries:
            raise ValueError("geometry %r is already registered" % (name,))
        kind, geo = wire.geometry_from_descriptor(descriptor)
        entry = GeometryEntry(kind, geo, geo.volume_shape, geo.detector_shape)
        self.geometries[name] = entry
        self.short_updates = max(e.updates for e in self.geometries.values()) // 8
        return entry

    def executor(self, cls: JobClass) -> Executor:
        if cls not in self.executors:
            self.executors[cls] = Executor(cls, self.geometries[cls.geometry], self.device, self.max_batch,
                                           self.use_graphs)
        return self.executors[cls]

    def warmup(self, classes, batch_sizes=(1,)) -> float:
        """Start-up work a server does before taking requests: the buffer sets
        of each class and the graphs of the given batch sizes, so that first
        requests do not pay allocation and capture.  Returns the seconds it
        took."""
        t0 = time.perf_counter()
        stream = self.streams[0]
        for cls in classes:
            ex = self.executor(cls)
            for b in batch_sizes:
                if b <= self.max_batch:
                    ex.prepare(b, stream)
        self.torch.cuda.synchronize(self.device)
        return time.perf_counter() - t0

    def free_hbm(self) -> int:
        """Free device memory, counting what torch's allocator holds unused."""
        torch = self.torch
        free, _ = torch.cuda.mem_get_info(self.device)
        return free + torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)

    def admit_memory(self, ex: Executor, bset: int, batch: int) -> bool:
        """Memory admission: the batch's result copies, and the buffer set if
        it is not resident yet, must fit the free HBM above the reserve;
        idle buffer sets of other classes are evicted (oldest first) to make
        room.  The device is asked for its free memory only when the budget
        left from the last answer cannot cover the request: the query
        (cudaMemGetInfo) can take tens of milliseconds, and asked for every
        batch it stalled the whole loop."""
        need = (ex.result_bytes(batch) if self.keep_results else 0) + (0 if ex.allocated(bset) else ex.set_bytes())
        if need == 0:
            return True
        if self._budget >= need:
            self._budget -= need
            return True
        free = self.free_hbm() - self.hbm_reserve
        if free >= need:
            self._budget = free - need
            return True
        idle = sorted(((e.last_use[i], e, i) for e in self.executors.values() if e is not ex
                       for i in range(e.n_sets) if e.allocated(i) and not e.busy[i]), key=lambda r: r[0])
        for _, e, i in idle:
            free += e.evict(i)
            self.evictions += 1
            if free >= need:
                self._budget = free - need
                return True
        self._budget = free
        return False

    def run_trace(self, jobs: List[Job], realtime: bool = True) -> ServeStats:
        """Serves jobs (sorted by arrival).  realtime=True replays arrivals on
        the wall clock; False admits every job as soon as capacity allows."""
        torch = self.torch
        pending = collections.deque(sorted(jobs, key=lambda j: j.arrival))
        ready: "collections.OrderedDict[JobClass, collections.deque]" = collections.OrderedDict()
        inflight = []  # (event, batch jobs, executor, buffer set, results)
        stream_i = 0
        t0 = self.clock()
        total_updates = 0

        def now():
            return self.clock() - t0

        while pending or ready or inflight:
            tnow = now()
            while pending and (not realtime or pending[0].arrival <= tnow):
                j = pending.popleft()
                ready.setdefault(j.cls, collections.deque()).append(j)
            # retire finished batches
            still = []
            for rec in inflight:
                ev, bjobs, ex, bset, results = rec
                if ev.query():
                    tdone = now()
                    for k, j in enumerate(bjobs):
                        j.result = results[k] if results else None
                        j.done = tdone
                        total_updates += j.updates
                    ex.busy[bset] = False
                    ex.last_use[bset] = tdone
                else:
                    still.append(rec)
            inflight = still
            # admit: oldest waiting class first, as many of its jobs as fit
            launched = False
            while ready and len(inflight) < self.max_inflight:
                # oldest waiting class whose executor has a free buffer set
                free = [c for c in ready if self.executor(c).free_set() is not None]
                if not free:
                    break
                cls = min(free, key=lambda c: ready[c][0].arrival)
                q = ready[cls]
                ex = self.executor(cls)
                bset = ex.free_set()
                b = min(len(q), self.max_batch)
                if not self.admit_memory(ex, bset, b):
                    if inflight:
                        break  # wait for a batch to retire
                    raise MemoryError("job class %s does not fit the free HBM" % (cls,))
                bjobs = [q.popleft() for _ in range(b)]
                if not q:
                    del ready[cls]
                short = self.geometries[cls.geometry].updates <= self.short_updates
                pool = self.fast_streams if short else self.streams
                stream = pool[stream_i % len(pool)]
                stream_i += 1
                inp, out, _ = ex.allocate(bset)
                ex.busy[bset] = True
                tadmit = now()
                with torch.cuda.stream(stream):
                    for k, j in enumerate(bjobs):
                        j.admit = tadmit
                        inp[k].copy_(j.data, non_blocking=True)
                ex.run(b, bset, stream)
                with torch.cuda.stream(stream):
                    # results stay on the device (copied out of the reused buffers)
                    results = [out[k].clone() for k in range(b)] if self.keep_results else None
                    ev = torch.cuda.Event()
                    ev.record(stream)
                inflight.append((ev, bjobs, ex, bset, results))
                self.batches += 1
                self.batch_sizes.append(b)
                launched = True
            if not launched and inflight:
                time.sleep(0)  # yield; completion is polled
            elif not launched and not inflight and pending and realtime:
                wait = pending[0].arrival - now()
                if wait > 0:
                    time.sleep(min(wait, 0.001))
        torch.cuda.synchronize(self.device)
        wall = now()
        # a bounded device wait that gave up leaves some result invalid
        from . import ops
        ops.check_device_errors(self.device)
        lat = np.array([(j.done - j.arrival) * 1e3 for j in jobs])
        replays = sum(ex.graph_replays for ex in self.executors.values())
        return ServeStats(lat, percentile(lat, 50), percentile(lat, 99), total_updates / wall / 1e9, wall,
                          self.batches, float(np.mean(self.batch_sizes)) if self.batch_sizes else 0.0, replays,
                          per_class_latency(jobs))


def run_plain(jobs: List[Job], geometries: Dict[str, GeometryEntry], device=None,
              clock: Callable[[], float] = time.perf_counter, realtime: bool = True,
              keep_results: bool = True) -> ServeStats:
    """The plain path: one job per launch, FP32, one stream, in arrival order,
    each job through the public op API (results kept on the device, or
    dropped after completion like the server's with keep_results=False)."""
    import torch

    from . import ops
    dev = torch.device(device or "cuda")
    t0 = clock()
    total = 0
    for j in sorted(jobs, key=lambda j: j.arrival):
        if realtime:
            while clock() - t0 < j.arrival:
                time.sleep(0.0002)
        e = geometries[j.cls.geometry]
        x = j.data.to(dev, non_blocking=True).float()[None]
        g = e.geo
        j.admit = clock() - t0
        if j.cls.op == "fan_fwd":
            r = ops.fan_projection2d(x, g.detector_shape, *g.args())
        elif j.cls.op == "fan_bp":
            r = ops.fan_backprojection2d(x, g.volume_shape, *g.args())
        elif j.cls.op == "cone_fwd":
            r = ops.cone_projection3d(x, g.detector_shape, *g.args())
        else:
            r = ops.cone_backprojection3d(x, g.volume_shape, *g.args())
        j.result = r[0] if keep_results else None
        torch.cuda.current_stream(dev).synchronize()
        j.done = clock() - t0
        total += j.updates
    torch.cuda.synchronize(dev)
    wall = clock() - t0
    lat = np.array([(j.done - j.arrival) * 1e3 for j in jobs])
    return ServeStats(lat, percentile(lat, 50), percentile(lat, 99), total / wall / 1e9, wall, len(jobs), 1.0, 0,
                      per_class_latency(jobs))


def job_from_request(req: dict, geometries: Dict[str, GeometryEntry], arrival: float = 0.0) -> Job:
    """A Job from a decoded wire request (wire.decode_request): the input in
    pinned host memory in its storage dtype, checked against the geometry."""
    import torch
    entry = geometries.get(req["geometry"])
    if entry is None:
        raise KeyError("unknown geometry %r" % (req["geometry"],))
    kind, direction = req["op"].split("_")
    if kind != entry.kind:
        raise ValueError("op %s on a %s geometry" % (req["op"], entry.kind))
    shape = entry.volume_shape if direction == "fwd" else entry.sinogram_shape
    data = np.asarray(req["data"])
    if tuple(data.shape) != tuple(shape):
        raise ValueError("input of shape %s, the geometry needs %s" % (data.shape, tuple(shape)))
    if req["dtype"] == "bf16":
        t = torch.from_numpy(data.astype(np.int16, copy=False)).view(torch.bfloat16)
    else:
        t = torch.from_numpy(np.array(data, copy=True))
    t = t.contiguous().pin_memory()
    return Job(int(req["id"]), JobClass(req["op"], req["geometry"], req["dtype"]), t, arrival, entry.updates)


def result_message(job: Job) -> bytes:
    """The job's result (device or host tensor) as a wire result message, in
    the dtype the server produced (FP32 volumes for backprojections)."""
    import torch
    from . import wire
    r = job.result.detach().cpu().contiguous()
    if r.dtype == torch.bfloat16:
        return wire.encode_result(job.id, "bf16", r.view(torch.int16).numpy().view(np.uint16))
    name = {torch.float32: "fp32", torch.float16: "fp16"}[r.dtype]
    return wire.encode_result(job.id, name, r.numpy())


def make_jobs(trace, geometries: Dict[str, GeometryEntry], seed: int = 0, pin: bool = True) -> List[Job]:
    """Materialises a trace with seeded inputs: phantoms for forward jobs,
    random non-negative sinograms for backprojections (host memory).  Inputs
    are shared per (geometry, op, dtype) to bound host memory."""
    import torch
    cache = {}
    jobs = []
    for i, (t, cls) in enumerate(trace):
        e = geometries[cls.geometry]
        dt = {"fp32": torch.float32, "bf16": torch.bfloat16, "fp16": torch.float16}[cls.dtype]
        key = (cls, seed)
        if key not in cache:
            rng = np.random.Generator(np.random.PCG64(zlib.crc32(("%s/%s/%d" % (cls.geometry, cls.op, seed)).encode())))
            if cls.op.endswith("_fwd"):
                if e.kind == "fan":
                    arr = _phantoms.ellipse_phantom_2d(e.volume_shape, e.geo.volume_spacing, seed=seed)[0]
                else:
                    sp = np.asarray(e.geo.volume_spacing, np.float64)
                    field = [e.volume_shape[k] * sp[k] for k in (2, 1, 0)]
                    ell = _phantoms.random_ellipsoids(seed, field, n=32)
                    arr = _phantoms.rasterise_ellipsoids_torch(ell, e.volume_shape, sp, e.geo.volume_origin,
                                                               "cuda").cpu().numpy()
            else:
                arr = rng.uniform(0.0, 1.0, e.sinogram_shape).astype(np.float32)
            ten = torch.from_numpy(np.ascontiguousarray(arr)).to(dt)
            cache[key] = ten.pin_memory() if pin else ten
        jobs.append(Job(i, cls, cache[key], t, e.updates))
    return jobs
