"""Serving loop: continuous batching of integrate and extract requests from
concurrent reconstruction sessions.

No counterpart in the reference (its arms integrate one volume per call).
One host thread drives one ``Batch`` (at most 64 attached sessions):

* Admission. A session waits from its first request until its footprint
  (table, voxel pool, update scratch, staging and mesh buffers, per
  ``footprint_bytes``) fits both the HBM budget ledger and the device's free
  memory (``torch.cuda.mem_get_info`` minus a headroom); sessions are
  admitted first come, first served. An admitted session's volume stays
  resident in HBM until its last request is done, then it is detached; its
  memory is freed when a waiting session needs the room (freeing synchronises
  the device, so it is not done while nothing waits).
* Continuous batching. Every step takes the oldest integrate request of each
  admitted session (one frame per session per step; a session's requests
  run in arrival order), copies the frames from pinned host memory on a
  copy stream into the session's other staging buffer (so the upload
  overlaps the step still running) and queues one batched step after the
  copies; at most ``max_inflight`` steps are on the GPU while the host forms
  the next, so requests that arrive during a step join the next one.
* Eviction. When a waiting session does not fit, admitted sessions with
  nothing queued or in flight are moved to host snapshots (least recently
  active first) and freed; an evicted session waits for admission again on
  its next request and is restored from its snapshot, exactly as it was.
* Extraction. A session whose oldest request is an extract, with none of
  its frames in flight, extracts its mesh into its device buffer on its own
  stream, concurrently with the batch steps of the other sessions.
* Latency. A request's latency is the time from its arrival to the moment
  the loop observes its step (or extraction) complete.

Results are those of integrating each session alone (the batched passes are
bit-identical to osn_tsdf_cuda_integrate), which the tests check.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import volume as _vol
from .batch import Batch
from .volume import CudaVolume

SCRATCH_SLOTS = 1 << 20
MESH_CAP_MAX = 1 << 26  # vertices; the extraction buffer doubles up to this on overflow


def mesh_capacity(spec) -> int:
    """Initial extraction buffer (vertices): a block crossed by a surface holds
    about 64 surface cubes of ~6 vertices each; sized for the pool, between 4
    vertices per point of the largest frame and 16M vertices. Allocating it at
    admission keeps allocation (a device-wide synchronisation) out of the
    serving loop; a mesh that does not fit doubles the buffer."""
    return int(min(max(spec.pool * 384, spec.max_points * 4), 1 << 24))


def footprint_bytes(spec, storage: int) -> int:
    """Device memory a session holds while admitted."""
    steps = max(1, math.ceil(spec.trunc / spec.voxel - 1e-9))
    per_voxel = {_vol.STORAGE_FP32: 20, _vol.STORAGE_FP16_U16: 4, _vol.STORAGE_FP64: 12}[storage]
    per_voxel += 4 + 8  # batch count and fixed-point sum
    n_records = spec.max_points * (2 * steps + 1)
    table = (spec.hash_slots + SCRATCH_SLOTS) * 16
    pool = spec.pool * (512 * per_voxel + 12 + 4 * 3)
    scratch = n_records * (4 + 4 + 8) + (n_records // 2 + 1) * 16
    stage = 2 * spec.max_points * 12  # double-buffered frame staging
    mesh = mesh_capacity(spec) * 24
    return int(table + pool + scratch + stage + mesh)


@dataclass
class Request:
    kind: str          # "integrate" or "extract"
    session: int
    frame: int         # integrate: frame index (into the session's frame list, cyclic)
    arrival: float     # seconds from the start of the run
    done: float = -1.0
    vertices: int = -1


@dataclass
class _Session:
    spec: object
    frames: list       # [(pinned host points (n, 3), cam)]
    queue: deque = field(default_factory=deque)
    vol: CudaVolume | None = None
    slot: int = -1
    stage: object = None      # two staging buffers, alternated per frame
    stage_ev: list = field(default_factory=lambda: [None, None])  # last step reading each
    flip: int = 0
    mesh: object = None
    inflight: int = 0
    remaining: int = 0  # requests not yet done
    footprint: int = 0
    admitted_at: float = -1.0
    closed: bool = False
    snapshot: object = None   # host copy while evicted
    last_active: float = 0.0
    evictions: int = 0


class Server:
    def __init__(self, budget_bytes: float = 120e9, storage: int = _vol.STORAGE_FP16_U16,
                 graph: bool = True, max_inflight: int = 2, headroom_bytes: float = 2e9,
                 shape=None, autotune_steps: int = 0, evict: bool = True):
        import torch
        self.torch = torch
        self.budget = float(budget_bytes)
        self.storage = storage
        self.headroom = float(headroom_bytes)
        self.max_inflight = max_inflight
        self.batch = Batch(64)
        self.batch.set_graph(graph)
        if shape is not None:
            self.batch.set_shape(*shape)
        self.autotune_steps = autotune_steps
        self.stream = torch.cuda.ExternalStream(self.batch.stream_handle())
        self.copy_stream = torch.cuda.Stream()  # frame uploads overlap the running step
        self.ledger = 0
        self.peak_ledger = 0
        self.peak_sessions = 0
        self.steps = 0
        self.keep_volumes = False  # tests keep finished volumes for comparison
        self.finished: dict[int, CudaVolume] = {}
        self.graveyard: list = []  # closed sessions' memory, freed lazily
        self.evict = evict          # snapshot idle sessions to host when others wait
        self.evictions = 0
        self.restores = 0

    # -- admission -----------------------------------------------------------
    def _try_admit(self, s: _Session, now: float) -> bool:
        if self.batch is None or len([x for x in self.sessions if x.vol is not None and not x.closed]) >= 64:
            return False
        fp = footprint_bytes(s.spec, self.storage)
        if self.ledger + fp > self.budget and self.graveyard:
            self._bury(fp)  # release finished sessions only when the room is needed
        if self.ledger + fp > self.budget and self.evict:
            self._evict_for(fp, now)
        if self.ledger + fp > self.budget:
            return False
        free, _ = self.torch.cuda.mem_get_info()
        if free < fp + self.headroom:
            return False
        sp = s.spec
        s.vol = CudaVolume(sp.voxel, sp.pool, sp.trunc, sp.cap, sp.hash_slots, storage=self.storage)
        if s.snapshot is not None:  # back from eviction
            s.vol.restore(s.snapshot)
            s.snapshot = None
            self.restores += 1
        s.slot = self.batch.add(s.vol, sp.max_points)
        s.inflight = 0
        s.stage_ev = [None, None]
        s.stage = [self.torch.empty((sp.max_points, 3), dtype=self.torch.float32, device="cuda")
                   for _ in range(2)]
        s.mesh = self.torch.empty((mesh_capacity(sp), 6), dtype=self.torch.float32, device="cuda")
        s.footprint = fp
        s.admitted_at = now
        self.ledger += fp
        self.peak_ledger = max(self.peak_ledger, self.ledger)
        live = sum(1 for x in self.sessions if x.vol is not None and not x.closed)
        self.peak_sessions = max(self.peak_sessions, live)
        return True

    def _evict_for(self, need: int, now: float) -> bool:
        """Move idle sessions (nothing queued or in flight) to host snapshots,
        least recently active first, until `need` bytes fit the budget."""
        idle = [x for x in self.sessions
                if x.vol is not None and not x.closed and not x.queue and not x.inflight and x.remaining]
        idle.sort(key=lambda x: x.last_active)
        for x in idle:
            if self.ledger + need <= self.budget:
                break
            self.batch.remove(x.slot)  # waits for the queued steps
            x.snapshot = x.vol.snapshot()
            x.vol.close()
            x.vol = None
            x.stage = x.mesh = None
            x.stage_ev = [None, None]
            self.ledger -= x.footprint
            x.evictions += 1
            self.evictions += 1
        return self.ledger + need <= self.budget

    def _extract(self, s: _Session) -> int:
        """Mesh into the session's device buffer; a full buffer is doubled
        (and charged to the ledger) until the mesh fits."""
        while True:
            n = s.vol.extract_mesh_device(s.mesh, None, s.mesh.shape[0], 0.5, 0.0)
            if n >= 0 or s.mesh.shape[0] >= MESH_CAP_MAX:
                return n
            grow = s.mesh.shape[0] * 24
            s.mesh = None
            s.mesh = self.torch.empty((2 * grow // 24, 6), dtype=self.torch.float32, device="cuda")
            s.footprint += grow
            self.ledger += grow
            self.peak_ledger = max(self.peak_ledger, self.ledger)

    def _close(self, s: _Session):
        """Detach a finished session. Its memory is released lazily: freeing
        multi-GB buffers synchronises the whole device, so the volume goes to
        a graveyard (still on the ledger) that is emptied only when a waiting
        session needs the room, or at the end of the run."""
        self.batch.remove(s.slot)
        if self.keep_volumes:
            self.finished[s.spec.index] = s.vol
        self.graveyard.append((s.vol, s.stage, s.mesh, s.footprint))
        s.stage = s.mesh = None
        s.stage_ev = [None, None]
        s.closed = True

    def _bury(self, need_bytes: float = float("inf")):
        """Free graveyard volumes (oldest first) until need_bytes fit the ledger."""
        while self.graveyard and self.ledger + need_bytes > self.budget:
            vol, stage, mesh, fp = self.graveyard.pop(0)
            if not self.keep_volumes:
                vol.close()
            del stage, mesh
            self.ledger -= fp

    # -- the loop ------------------------------------------------------------
    def run(self, specs, frames, requests: list[Request], realtime: bool = True,
            open_first: bool = False) -> dict:
        """Serve `requests` (sorted or not) for sessions `specs` whose frames
        are `frames[i]` (host (n, 3) float32 arrays and cams; frame k of a
        request uses frames[i][k % len]). realtime: requests become visible at
        their arrival time; otherwise all at once (throughput at saturation).
        open_first: the sessions open before the first frame arrives, so every
        session that fits is admitted before the clock starts (the time this
        takes is reported as open_s); the rest wait for memory as usual."""
        torch = self.torch
        reqs = sorted(requests, key=lambda r: r.arrival)
        self.sessions = []
        for sp, fr in zip(specs, frames):
            pinned = [(torch.from_numpy(np.ascontiguousarray(p)).pin_memory(), cam) for p, cam in fr]
            self.sessions.append(_Session(spec=sp, frames=pinned))
        for r in reqs:
            self.sessions[r.session].remaining += 1
        waiting: deque[_Session] = deque()
        inflight: deque = deque()  # (event, [requests])
        self.t_tuned = 0.0
        self.t_admitted = 0.0  # last admission
        self.open_s = 0.0
        if open_first:
            t_open = time.perf_counter()
            for sess in self.sessions:
                if not self._try_admit(sess, 0.0):
                    break  # first come, first served: later sessions wait their turn
            self.batch.synchronize()
            self.open_s = time.perf_counter() - t_open
        nxt = 0
        t0 = time.perf_counter()
        tuned = self.autotune_steps <= 0
        while nxt < len(reqs) or any(not s.closed and s.remaining for s in self.sessions) or inflight:
            now = time.perf_counter() - t0
            # Arrivals.
            while nxt < len(reqs) and (not realtime or reqs[nxt].arrival <= now):
                r = reqs[nxt]
                if not realtime:
                    r.arrival = now
                s = self.sessions[r.session]
                if s.vol is None and not s.closed and not s.queue and s not in waiting:
                    waiting.append(s)
                s.queue.append(r)
                nxt += 1
            # Admission, first come first served.
            while waiting and self._try_admit(waiting[0], now):
                waiting.popleft()
                self.t_admitted = now
            # Completed steps.
            while inflight and inflight[0][0].query():
                _, rs = inflight.popleft()
                t = time.perf_counter() - t0
                for r in rs:
                    r.done = t
                    s = self.sessions[r.session]
                    s.inflight -= 1
                    s.remaining -= 1
                    s.last_active = t
            # Extractions of sessions with nothing in flight.
            for s in self.sessions:
                if s.vol is None or s.closed or s.inflight or not s.queue or s.queue[0].kind != "extract":
                    continue
                r = s.queue.popleft()
                r.vertices = self._extract(s)
                r.done = time.perf_counter() - t0
                s.remaining -= 1
                s.last_active = r.done
            # Sessions with every request done leave; their memory admits others.
            for s in self.sessions:
                if s.vol is not None and not s.closed and s.remaining == 0 and not s.queue:
                    self._close(s)
            # Next step: the oldest integrate request of every admitted session.
            if len(inflight) < self.max_inflight:
                members, used = [], []
                with torch.cuda.stream(self.copy_stream):
                    for s in self.sessions:
                        if s.vol is None or s.closed or not s.queue or s.queue[0].kind != "integrate":
                            continue
                        r = s.queue.popleft()
                        host, cam = s.frames[r.frame % len(s.frames)]
                        n = host.shape[0]
                        buf = s.flip
                        s.flip ^= 1
                        if s.stage_ev[buf] is not None:  # the step that last read it
                            self.copy_stream.wait_event(s.stage_ev[buf])
                        s.stage[buf][:n].copy_(host, non_blocking=True)
                        self.batch.set_frame(s.slot, s.stage[buf][:n], cam)
                        s.inflight += 1
                        members.append(r)
                        used.append((s, buf))
                if members:
                    copied = torch.cuda.Event()
                    copied.record(self.copy_stream)
                    self.stream.wait_event(copied)
                    if not tuned:
                        self.batch.autotune(self.autotune_steps)
                        tuned = True
                    self.batch.step()
                    ev = torch.cuda.Event()
                    ev.record(self.stream)
                    for s, buf in used:
                        s.stage_ev[buf] = ev
                    inflight.append((ev, members))
                    self.steps += 1
                    if self.steps == 16 * max(self.autotune_steps, 0):
                        self.t_tuned = time.perf_counter() - t0
                    continue
            if inflight:
                inflight[0][0].synchronize() if not realtime else time.sleep(0)
            elif realtime and nxt < len(reqs):
                wait = reqs[nxt].arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.0005))
        self.batch.synchronize()
        t_end = time.perf_counter() - t0
        self._bury()
        return self._stats(reqs, t_end)

    def _stats(self, reqs, t_end) -> dict:
        integ = [r for r in reqs if r.kind == "integrate"]
        ext = [r for r in reqs if r.kind == "extract"]

        def pct(xs, q):
            return float(np.percentile(np.asarray(xs) * 1e3, q)) if xs else None

        lat_i = [r.done - r.arrival for r in integ]
        lat_e = [r.done - r.arrival for r in ext]
        # Steady state: arrivals after start-up (autotuning steps, and the
        # admissions of sessions that arrived together at the start).
        start = max(self.t_tuned, min(self.t_admitted, 1.0))
        lat_s = [r.done - r.arrival for r in integ if r.arrival >= start]
        first = min((r.arrival for r in reqs), default=0.0)
        last = max((r.done for r in reqs), default=0.0)
        return {
            "frames": len(integ), "extracts": len(ext), "steps": self.steps,
            "frames_per_s": len(integ) / max(last - first, 1e-9),
            "frames_per_step": len(integ) / max(self.steps, 1),
            "integrate_latency_ms": {"p50": pct(lat_i, 50), "p99": pct(lat_i, 99), "max": pct(lat_i, 100)},
            "integrate_latency_ms_steady": {"p50": pct(lat_s, 50), "p99": pct(lat_s, 99),
                                            "from_s": start, "requests": len(lat_s)},
            "extract_latency_ms": {"p50": pct(lat_e, 50), "p99": pct(lat_e, 99)},
            "wall_s": t_end, "open_s": self.open_s, "peak_sessions": self.peak_sessions,
            "evictions": self.evictions, "restores": self.restores,
            "peak_ledger_gb": self.peak_ledger / 1e9, "budget_gb": self.budget / 1e9,
            "shape": self.batch.shape(),
        }

    def close(self):
        """Detach and free every session, then the batch (torch buffers used on
        the batch's stream go before the stream does)."""
        if getattr(self, "batch", None) is None:
            return
        self.batch.synchronize()
        for s in getattr(self, "sessions", []):
            if s.vol is not None and not s.closed:
                self._close(s)
            s.frames = []
            s.stage = s.mesh = None
            s.stage_ev = [None, None]
        self.sessions = []
        self._bury()
        self.torch.cuda.synchronize()
        self.batch.close()
        self.batch = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def poisson_schedule(specs, rate_fps: float, extract_every: int, seed: int = 7) -> list[Request]:
    """Integrate requests of every session as independent Poisson streams whose
    rates sum to rate_fps (while all sessions are active); an extract request
    right after every extract_every-th frame of a session."""
    rng = np.random.default_rng(seed)
    per = rate_fps / len(specs)
    out = []
    for sp in specs:
        t = 0.0
        for k in range(sp.frames):
            t += rng.exponential(1.0 / per)
            out.append(Request("integrate", sp.index, k, t))
            if extract_every and (k + 1) % extract_every == 0:
                out.append(Request("extract", sp.index, k, t + 1e-9))
    return out
