"""Continuous-batching stereo server on one GPU.

Camera streams are opened once.  Each stream owns a solver handle whose device state (pyramid,
vector fields, mask, the solver buffers whose stale values the reference carries between frames,
and, with warm starts, the previous disparity) stays on the GPU between its frames.

Requests (one stereo pair of a stream) queue on the host.  The server runs ``lanes`` batch slots,
each with its own CUDA stream.  Whenever a slot is free it takes up to ``max_batch`` waiting
requests, at most one per camera (a camera's frames are solved in order), and launches them as
one batched fused solve that overlaps the batches already on the GPU.  Finished slots are
detected by event, their disparities copied back, and their requests' latencies recorded.  A
request therefore joins the next free slot without waiting for the batches in flight.

Admission by free device memory happens per request, as slots and memory free up:
* a request is launched only when the device memory it still needs fits in the free memory
  less ``reserve_bytes`` (its stream's state if the stream is parked, the fused buffers on a
  stream's first fused solve, and its image and disparity buffers); otherwise it waits;
* to make room, the server parks idle streams, least recently used first: their state is
  exported to page-locked host memory (``vfs_export_state``) and their device memory freed;
  a parked stream's next request brings the state back (``vfs_import_state``), and the stream
  continues bit for bit where it stopped.
Opening a stream allocates its state the same way (parking idle streams if needed) and is refused
with AdmissionError when even that leaves no room; a request that cannot fit with every other
stream parked raises AdmissionError instead of waiting for ever.

Each pair's solve reads only its own state, so a stream's results are the same whether it is
served alone, in a mix, or parked in between (``tests/test_gpu_serving.py``).
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field
from typing import Deque, Dict, List, Optional

import numpy as np

from ._native import lib
from .stereotgv import StereoBatch, StereoTgv


class AdmissionError(RuntimeError):
    """A stream cannot be admitted: its footprint does not fit beside the reserve."""


@dataclass
class Request:
    stream_id: int
    seq: int
    i0: np.ndarray
    i1: np.ndarray
    t_submit: float
    t_launch: float = 0.0
    t_done: float = 0.0
    u: Optional[np.ndarray] = None
    cancelled: bool = False

    @property
    def latency_ms(self) -> float:
        return 1000.0 * (self.t_done - self.t_submit)


@dataclass
class _Camera:
    stream_id: int
    width: int
    height: int
    n_levels: int
    params: dict
    mask: np.ndarray
    tv: np.ndarray
    cv: np.ndarray
    warm_level: int
    solver: Optional[StereoTgv] = None   # None while parked
    parked_state: Optional[object] = None  # page-locked host copy of the state while parked
    busy: bool = False
    frames: int = 0
    last_used: float = 0.0
    fused_ready: bool = False  # its fused buffers exist (allocated on the first fused solve)


@dataclass
class _Lane:
    stream: object
    batch: StereoBatch
    event: object = None
    requests: List[Request] = field(default_factory=list)
    ins: list = field(default_factory=list)
    outs: list = field(default_factory=list)
    hosts: list = field(default_factory=list)
    # buffers reused from batch to batch: shape -> list of page-locked (i0, i1, u) host tensors
    # followed by their device counterparts
    pinned: Dict[tuple, list] = field(default_factory=dict)

    @property
    def busy(self) -> bool:
        return self.event is not None


DEFAULT_PARAMS = dict(beta=10.0, gamma=0.8, alpha0=17.0, alpha1=1.2, timestep_lambda=1.0, lambda_=5.0, fScale=2.0,
                      nWarpIters=3, nSolverIters=50, limitRange=0.1)


class StereoServer:
    def __init__(self, device: int = 0, max_batch: int = 8, lanes: int = 2, half_storage: bool = True,
                 reserve_bytes: int = 1 << 30, use_graph: bool = True, path: str = "fused"):
        """path="plain" serves one request at a time with the drop-in path (the baseline)."""
        import torch
        self.torch = torch
        self.device = torch.device("cuda", device)
        torch.cuda.set_device(self.device)
        self.path = path
        if path == "plain":
            max_batch, half_storage = 1, False
        self.max_batch = max_batch
        self.half = half_storage
        self.reserve = reserve_bytes
        self.cameras: Dict[int, _Camera] = {}
        self.queue: Deque[Request] = collections.deque()
        self.lanes = []
        for _ in range(lanes):
            b = StereoBatch(half_storage=half_storage)
            b.set_graph(use_graph)
            b.set_autotune(False)  # no timing passes (host synchronisations) inside the serving loop
            # latency first: every request of a batch runs its full-resolution level at once
            # (a full-resolution limit raises throughput but delays the later pairs of a batch)
            b.set_fine_concurrency(0)
            st = torch.cuda.Stream(device=self.device)
            b.set_stream(st)
            self.lanes.append(_Lane(stream=st, batch=b))
        self.done: List[Request] = []
        self._seq = 0
        self.counters = collections.Counter()  # deferred admissions, parks, unparks, cancels
        self._free_val: Optional[int] = None
        self._free_reserved = 0

    # ---- memory -----------------------------------------------------------------------
    def _free(self, fresh: bool = False) -> int:
        """Free device memory.  The driver's figure (cudaMemGetInfo) took up to 195 ms per query
        while the GPU was busy, so it is read only when the server's own allocations or releases
        of stream state have made the last reading stale, when a request does not fit by the
        last reading, or when `fresh`; in between, memory the framework's caching allocator has
        reserved since the reading is taken off it.  Memory that another process takes in
        between is seen at the next reading."""
        torch = self.torch
        reserved = int(torch.cuda.memory_reserved(self.device))
        if fresh or self._free_val is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            self._free_val, self._free_reserved = int(free), reserved
        return self._free_val - max(0, reserved - self._free_reserved)

    def _forget_free(self) -> None:
        self._free_val = None

    def _state_bytes(self, cam: _Camera, fused: bool) -> int:
        return int(lib().vfs_estimate_device_bytes(cam.width, cam.height, cam.n_levels, cam.params["fScale"], 32,
                                                   1 if fused else 0))

    def _request_bytes(self, cam: _Camera) -> int:
        """Device memory a request of this camera still needs before it can run."""
        need = 2 * cam.width * cam.height + 4 * cam.width * cam.height  # images and disparity
        if cam.solver is None:
            need += self._state_bytes(cam, self.path != "plain" and cam.fused_ready)
        if self.path != "plain" and not cam.fused_ready:
            need += self._state_bytes(cam, True) - self._state_bytes(cam, False)
        return need

    def footprint(self, width: int, height: int, n_levels: int, f_scale: float = 2.0) -> int:
        return int(lib().vfs_estimate_device_bytes(width, height, n_levels, f_scale, 32, 1))

    # ---- streams --------------------------------------------------------------------
    def open_stream(self, stream_id: int, width: int, height: int, mask, tv, cv, n_levels: int,
                    params: Optional[dict] = None, warm_start_level: int = -1) -> None:
        """Admit a camera stream and allocate its state, parking idle streams if that makes
        room.  warm_start_level >= 0: each frame after the first starts from the previous
        disparity at that pyramid level (vfs_set_warm_start)."""
        if stream_id in self.cameras:
            raise ValueError(f"stream {stream_id} already open")
        p = dict(DEFAULT_PARAMS, **(params or {}))
        cam = _Camera(stream_id, width, height, n_levels, p, np.ascontiguousarray(mask, np.float32),
                      np.ascontiguousarray(tv, np.float32), np.ascontiguousarray(cv, np.float32), int(warm_start_level))
        need = self._state_bytes(cam, False)
        if need == 0:
            raise AdmissionError(f"stream {stream_id}: invalid geometry")
        if not self._ensure_room(need, keep=set()):
            raise AdmissionError(f"stream {stream_id}: needs {need} bytes + reserve {self.reserve}, "
                                 f"free {self._free()}")
        cam.solver = self._new_solver(cam)
        cam.solver.copyMaskToDevice(cam.mask)
        cam.solver.loadVectorFields(cam.tv, cam.cv)
        cam.last_used = time.perf_counter()
        self.cameras[stream_id] = cam
        # staging (page-locked and device) for as many frames of this size as a batch can hold:
        # allocating it inside the serving loop stalled the loop for up to 113 ms while the GPU
        # was busy
        n = sum(1 for c in self.cameras.values() if (c.height, c.width) == (height, width))
        for lane in self.lanes:
            self._staging(lane, height, width, min(n, self.max_batch) - 1)

    def _new_solver(self, cam: _Camera) -> StereoTgv:
        self._forget_free()
        p = cam.params
        s = StereoTgv()
        s.set_solve_path(self.path != "plain", self.half)
        s.limitRange = p["limitRange"]
        s.initialize(cam.width, cam.height, p["beta"], p["gamma"], p["alpha0"], p["alpha1"], p["timestep_lambda"],
                     p["lambda_"], cam.n_levels, p["fScale"], p["nWarpIters"], p["nSolverIters"])
        if cam.warm_level >= 0:
            s.set_warm_start(cam.warm_level)
        return s

    def _release_solver(self, cam: _Camera) -> None:
        for lane in self.lanes:  # idle batches still list their last members
            if not lane.busy:
                lane.batch.clear()
        cam.solver.close()
        cam.solver = None
        self._forget_free()

    def park_stream(self, stream_id: int) -> None:
        """Move an idle stream's state to page-locked host memory and free its device memory."""
        cam = self.cameras[stream_id]
        if cam.solver is None:
            return
        if cam.busy:
            raise RuntimeError(f"stream {stream_id} has a frame in flight")
        n = int(lib().vfs_state_bytes(cam.solver.handle))
        host = self.torch.empty(n, dtype=self.torch.uint8).pin_memory()
        st = lib().vfs_export_state(cam.solver.handle, host.data_ptr(), n)
        if st != 0:
            raise RuntimeError(f"stream {stream_id}: export failed ({st})")
        cam.parked_state = host
        self._release_solver(cam)
        self.counters["parks"] += 1

    def _unpark(self, cam: _Camera) -> None:
        s = self._new_solver(cam)
        host = cam.parked_state
        st = lib().vfs_import_state(s.handle, host.data_ptr(), host.numel())
        if st != 0:
            s.close()
            raise RuntimeError(f"stream {cam.stream_id}: import failed ({st})")
        cam.solver = s
        cam.parked_state = None
        self.counters["unparks"] += 1

    def _ensure_room(self, need: int, keep: set) -> bool:
        """Park idle streams (least recently used first, those with waiting requests last)
        until `need` bytes fit beside the reserve."""
        if need + self.reserve <= self._free():
            return True
        if need + self.reserve <= self._free(fresh=True):
            return True
        self.torch.cuda.empty_cache()  # memory torch keeps cached is not free to the driver
        if need + self.reserve <= self._free(fresh=True):
            return True
        waiting = {r.stream_id for r in self.queue}
        idle = [c for c in self.cameras.values()
                if c.solver is not None and not c.busy and c.stream_id not in keep]
        idle.sort(key=lambda c: (c.stream_id in waiting, c.last_used))
        for c in idle:
            self.park_stream(c.stream_id)
            self.torch.cuda.synchronize(self.device)
            if need + self.reserve <= self._free(fresh=True):
                return True
        return need + self.reserve <= self._free(fresh=True)

    def close_stream(self, stream_id: int) -> None:
        """Close a stream between its frames; its waiting requests are cancelled."""
        cam = self.cameras.get(stream_id)
        if cam is None:
            return
        if cam.busy:
            raise RuntimeError(f"stream {stream_id} has a frame in flight")
        for r in [r for r in self.queue if r.stream_id == stream_id]:
            self.cancel(r)
        if cam.solver is not None:
            cam.solver.synchronize()
            self._release_solver(cam)
        del self.cameras[stream_id]

    # ---- requests -------------------------------------------------------------------
    def submit(self, stream_id: int, i0: np.ndarray, i1: np.ndarray, t_submit: Optional[float] = None) -> Request:
        if stream_id not in self.cameras:
            raise KeyError(f"stream {stream_id} not open")
        r = Request(stream_id, self._seq, i0, i1, time.perf_counter() if t_submit is None else t_submit)
        self._seq += 1
        self.queue.append(r)
        return r

    def cancel(self, request: Request) -> bool:
        """Withdraw a request that has not been launched yet; False if it already runs or ran."""
        try:
            self.queue.remove(request)
        except ValueError:
            return False
        request.cancelled = True
        self.counters["cancelled"] += 1
        return True

    def pending(self) -> int:
        return len(self.queue) + sum(len(l.requests) for l in self.lanes)

    def _harvest(self) -> List[Request]:
        fin = []
        for lane in self.lanes:
            if lane.busy and lane.event.query():
                now = time.perf_counter()
                for r, h in zip(lane.requests, lane.hosts):
                    r.u = h.numpy().copy()
                    r.t_done = now
                    cam = self.cameras.get(r.stream_id)
                    if cam is not None:
                        cam.busy = False
                        cam.frames += 1
                        cam.last_used = now
                    fin.append(r)
                lane.event = None
                lane.requests, lane.ins, lane.outs, lane.hosts = [], [], [], []
        self.done.extend(fin)
        return fin

    def _admit(self) -> List[Request]:
        """Pick up to max_batch waiting requests (one per camera, in arrival order) whose device
        memory fits, parking idle streams to make room; the others keep waiting."""
        picked, seen, committed = [], set(), 0
        for r in list(self.queue):
            if len(picked) >= self.max_batch:
                break
            cam = self.cameras[r.stream_id]
            if cam.busy or r.stream_id in seen:
                continue  # a camera's frames run in order: at most one in flight
            need = self._request_bytes(cam)
            if not self._ensure_room(committed + need, keep=seen | {r.stream_id}):
                self.counters["deferred"] += 1
                continue
            if cam.solver is None:
                self._unpark(cam)
                need = self._request_bytes(cam)  # the state is resident now
            committed += need
            picked.append(r)
            seen.add(r.stream_id)
        for r in picked:
            self.queue.remove(r)
        return picked

    def _staging(self, lane: _Lane, h: int, w: int, k: int):
        """The k-th buffer set of a lane for h x w frames: page-locked (i0, i1, u) and the
        device (i0, i1, u) the batch reads and writes.  A lane reuses them only once its
        previous batch has completed."""
        pool = lane.pinned.setdefault((h, w), [])
        torch = self.torch
        while len(pool) <= k:
            with torch.cuda.stream(lane.stream):  # device blocks of the lane's stream
                pool.append((torch.empty((h, w), dtype=torch.uint8).pin_memory(),
                             torch.empty((h, w), dtype=torch.uint8).pin_memory(),
                             torch.empty((h, w), dtype=torch.float32).pin_memory(),
                             torch.empty((h, w), dtype=torch.uint8, device=self.device),
                             torch.empty((h, w), dtype=torch.uint8, device=self.device),
                             torch.empty((h, w), dtype=torch.float32, device=self.device)))
        return pool[k]

    def _launch(self, lane: _Lane) -> bool:
        torch = self.torch
        picked = self._admit()
        if not picked:
            return False
        st = lane.stream
        lane.batch.clear()
        now = time.perf_counter()
        used = collections.Counter()
        with torch.cuda.stream(st):
            ins, outs, hosts = [], [], []
            for r in picked:
                cam = self.cameras[r.stream_id]
                cam.busy = True
                cam.solver.set_stream(st)
                key = (cam.height, cam.width)
                hi0, hi1, hu, di0, di1, du = self._staging(lane, cam.height, cam.width, used[key])
                used[key] += 1
                np.copyto(hi0.numpy(), r.i0)
                np.copyto(hi1.numpy(), r.i1)
                di0.copy_(hi0, non_blocking=True)
                di1.copy_(hi1, non_blocking=True)
                ins.append((di0, di1))
                outs.append(du)
                hosts.append(hu)
                if self.path != "plain":
                    lane.batch.add(cam.solver)
                r.t_launch = now
            if self.path == "plain":
                solver = self.cameras[picked[0].stream_id].solver
                solver.copy_images_from_device(*ins[0])
                solver.solveStereoForwardMasked()
                solver.copy_1d_disparity_to_device(outs[0])
            else:
                # each request's copies and solve on its own lane of the batch
                lane.batch.solve_device(ins, outs)
            for out, hu in zip(outs, hosts):
                hu.copy_(out, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(st)
        for r in picked:
            cam = self.cameras[r.stream_id]
            if not cam.fused_ready and self.path != "plain":
                self._forget_free()  # the first fused solve allocates the fused state
            cam.fused_ready = self.path != "plain"
        lane.ins, lane.outs, lane.hosts = ins, outs, hosts  # kept alive until the batch completes
        lane.event = ev
        lane.requests = picked
        return True

    def step(self) -> List[Request]:
        """One scheduling pass: collect finished batches, launch waiting requests on free slots."""
        fin = self._harvest()
        launched = False
        for lane in self.lanes:
            if not lane.busy and self.queue:
                launched = self._launch(lane) or launched
        if self.queue and not launched and not any(l.busy for l in self.lanes):
            # nothing runs and nothing could be admitted: no memory will free up by waiting
            r = self.queue[0]
            raise AdmissionError(f"request {r.seq} of stream {r.stream_id} does not fit in free device memory "
                                 f"beside the reserve even with every other stream parked")
        return fin

    def run_until_idle(self, poll_s: float = 0.0002) -> None:
        while self.pending():
            self.step()
            if self.pending():
                time.sleep(poll_s)

    # ---- statistics -----------------------------------------------------------------
    def stats(self, since: float = 0.0) -> dict:
        d = [r for r in self.done if r.t_submit >= since]
        out = {k: int(v) for k, v in self.counters.items()}
        if not d:
            out["frames"] = 0
            return out
        lat = np.array([r.latency_ms for r in d])
        span = max(r.t_done for r in d) - min(r.t_submit for r in d)
        out.update({"frames": len(d), "frames_per_s": len(d) / span if span > 0 else None,
                    "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                    "mean_ms": float(lat.mean())})
        return out


def poisson_schedule(rates: Dict[int, float], n_frames: Dict[int, int], seed: int = 0):
    """Arrival times (seconds from 0) of every stream's frames, Poisson with the given rates;
    returns a time-ordered list of (t, stream_id, frame_index)."""
    rng = np.random.default_rng(seed)
    ev = []
    for sid, rate in rates.items():
        t = 0.0
        for k in range(n_frames[sid]):
            t += rng.exponential(1.0 / rate)
            ev.append((t, sid, k))
    ev.sort()
    return ev


def replay(server: StereoServer, schedule, frames, realtime: bool = True, poll_s: float = 0.0002):
    """Submit scheduled frames (frames[sid][k] = (i0, i1)) at their arrival times while
    serving; returns the requests in submission order."""
    t0 = time.perf_counter()
    reqs = []
    idx = 0
    while idx < len(schedule) or server.pending():
        now = time.perf_counter() - t0
        while idx < len(schedule) and (not realtime or schedule[idx][0] <= now):
            t, sid, k = schedule[idx]
            i0, i1 = frames[sid][k]
            reqs.append(server.submit(sid, i0, i1, t_submit=t0 + (t if realtime else now)))
            idx += 1
        server.step()
        if server.pending() or idx < len(schedule):
            time.sleep(poll_s)
    return reqs
