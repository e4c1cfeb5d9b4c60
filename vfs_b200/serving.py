"""Continuous-batching stereo server on one GPU.

Camera streams are opened once. Each stream owns a solver handle whose device state
(pyramid, vector fields, mask and the solver buffers whose stale values the reference
carries between frames) stays on the GPU between its frames. A stream is admitted only when
its device footprint (``vfs_estimate_device_bytes``) plus a reserve fits in the free device
memory.

Requests (one stereo pair of a stream) queue on the host. The server runs ``lanes`` batch
slots, each with its own CUDA stream. Whenever a slot is free it takes up to ``max_batch``
waiting requests, at most one per camera (a camera's frames are solved in order), and
launches them as one batched fused solve. The launch overlaps the batches already on the
GPU. Finished slots are detected by event, their disparities copied back, and their requests'
latencies recorded. A request therefore joins the next free slot without waiting for the
batches in flight.

Each pair's solve reads only its own state, so a stream's results are the same whether it is
served alone or in a mix (``tests/test_gpu_serving.py``).
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
    """A stream cannot be admitted: not enough free device memory."""


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

    @property
    def latency_ms(self) -> float:
        return 1000.0 * (self.t_done - self.t_submit)


@dataclass
class _Camera:
    stream_id: int
    width: int
    height: int
    solver: StereoTgv
    busy: bool = False
    frames: int = 0


@dataclass
class _Lane:
    stream: object
    batch: StereoBatch
    event: object = None
    requests: List[Request] = field(default_factory=list)
    ins: list = field(default_factory=list)
    outs: list = field(default_factory=list)
    hosts: list = field(default_factory=list)

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

    # ---- streams --------------------------------------------------------------------
    def footprint(self, width: int, height: int, n_levels: int, f_scale: float = 2.0) -> int:
        return int(lib().vfs_estimate_device_bytes(width, height, n_levels, f_scale, 32, 1))

    def open_stream(self, stream_id: int, width: int, height: int, mask, tv, cv, n_levels: int,
                    params: Optional[dict] = None) -> None:
        """Admit a camera stream: allocate its handle if its footprint fits in free memory."""
        if stream_id in self.cameras:
            raise ValueError(f"stream {stream_id} already open")
        p = dict(DEFAULT_PARAMS, **(params or {}))
        need = int(lib().vfs_estimate_device_bytes(width, height, n_levels, p["fScale"], 32,
                                                   0 if self.path == "plain" else 1))
        free, _ = self.torch.cuda.mem_get_info(self.device)
        if need == 0 or need + self.reserve > free:
            raise AdmissionError(f"stream {stream_id}: needs {need} bytes + reserve {self.reserve}, free {free}")
        s = StereoTgv()
        s.set_solve_path(self.path != "plain", self.half)
        s.limitRange = p["limitRange"]
        s.initialize(width, height, p["beta"], p["gamma"], p["alpha0"], p["alpha1"], p["timestep_lambda"],
                     p["lambda_"], n_levels, p["fScale"], p["nWarpIters"], p["nSolverIters"])
        s.copyMaskToDevice(mask)
        s.loadVectorFields(tv, cv)
        self.cameras[stream_id] = _Camera(stream_id, width, height, s)

    def close_stream(self, stream_id: int) -> None:
        cam = self.cameras.get(stream_id)
        if cam is None:
            return
        if cam.busy:
            raise RuntimeError(f"stream {stream_id} has a frame in flight")
        cam.solver.synchronize()
        del self.cameras[stream_id]

    # ---- requests -------------------------------------------------------------------
    def submit(self, stream_id: int, i0: np.ndarray, i1: np.ndarray, t_submit: Optional[float] = None) -> Request:
        if stream_id not in self.cameras:
            raise KeyError(f"stream {stream_id} not open")
        r = Request(stream_id, self._seq, i0, i1, time.perf_counter() if t_submit is None else t_submit)
        self._seq += 1
        self.queue.append(r)
        return r

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
                    cam = self.cameras[r.stream_id]
                    cam.busy = False
                    cam.frames += 1
                    fin.append(r)
                lane.event = None
                lane.requests, lane.ins, lane.outs, lane.hosts = [], [], [], []
        self.done.extend(fin)
        return fin

    def _launch(self, lane: _Lane) -> bool:
        torch = self.torch
        picked, seen = [], set()
        rest = collections.deque()
        while self.queue and len(picked) < self.max_batch:
            r = self.queue.popleft()
            cam = self.cameras[r.stream_id]
            if cam.busy or r.stream_id in seen:
                rest.append(r)  # a camera's frames run in order: at most one in flight
                continue
            picked.append(r)
            seen.add(r.stream_id)
        rest.extend(self.queue)
        self.queue = rest
        if not picked:
            return False
        st = lane.stream
        lane.batch.clear()
        now = time.perf_counter()
        with torch.cuda.stream(st):
            ins, outs = [], []
            for r in picked:
                cam = self.cameras[r.stream_id]
                cam.busy = True
                cam.solver.set_stream(st)
                a = torch.from_numpy(np.ascontiguousarray(r.i0)).pin_memory().to(self.device, non_blocking=True)
                b = torch.from_numpy(np.ascontiguousarray(r.i1)).pin_memory().to(self.device, non_blocking=True)
                ins.append((a, b))
                outs.append(torch.empty((cam.height, cam.width), dtype=torch.float32, device=self.device))
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
            for out in outs:
                host = torch.empty(out.shape, dtype=torch.float32, pin_memory=True)
                host.copy_(out, non_blocking=True)
                lane.outs.append(out)
                lane.hosts.append(host)
            lane.ins = ins  # kept alive until the batch completes
            ev = torch.cuda.Event()
            ev.record(st)
        lane.event = ev
        lane.requests = picked
        return True

    def step(self) -> List[Request]:
        """One scheduling pass: collect finished batches, launch waiting requests on free slots."""
        fin = self._harvest()
        for lane in self.lanes:
            if not lane.busy and self.queue:
                self._launch(lane)
        return fin

    def run_until_idle(self, poll_s: float = 0.0002) -> None:
        while self.pending():
            self.step()
            if self.pending():
                time.sleep(poll_s)

    # ---- statistics -----------------------------------------------------------------
    def stats(self, since: float = 0.0) -> dict:
        d = [r for r in self.done if r.t_submit >= since]
        if not d:
            return {"frames": 0}
        lat = np.array([r.latency_ms for r in d])
        span = max(r.t_done for r in d) - min(r.t_submit for r in d)
        return {"frames": len(d), "frames_per_s": len(d) / span if span > 0 else None,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "mean_ms": float(lat.mean())}


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
