"""Continuous-batching MMFF optimisation service on one GPU.

Requests (one molecule x k conformers, MMFF94 or MMFF94s) arrive at any
time.  A scheduler thread

* prepares each request on the host (term extraction, packing -- a small
  thread pool, so preparation overlaps the GPU),
* admits prepared requests while the device-memory budget allows (tables,
  coordinates, results and optimizer scratch of the request, estimated
  before admission), each on its own CUDA stream from a pool, so requests
  that arrive while others are on the GPU start as soon as memory frees and
  run concurrently with them,
* keeps every admitted request's coordinates and optimizer state resident
  on the device until its kernel finishes, then copies the results back and
  completes the request's future.

Every request is one launch of the optimizer kernel whose instance (CTA
size, register-cached Hessian columns, shared- or global-memory Hessian)
depends only on that molecule's atom count, and the kernel is deterministic,
so a request's result is bit-for-bit the same alone or in any mix.
Molecules of 150 atoms or more use L-BFGS (m = 8), smaller ones dense BFGS.
"""
from __future__ import annotations

import queue
import threading
import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import mmff_minimize as mm
from .mmff_params import extract_mmff_params


@dataclass
class RequestResult:
    request_id: int
    positions: np.ndarray          # (k, N, 3) float32
    energies: np.ndarray           # (k,) float64
    status: np.ndarray             # (k,) int32
    converged: np.ndarray          # (k,) bool
    t_submit: float
    t_admit: float
    t_done: float

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


@dataclass
class _Req:
    rid: int
    mol: object
    positions: np.ndarray
    variant: str
    max_iters: int
    t_submit: float
    future: Future
    prep: Optional[Future] = None
    params: object = None
    nbytes: int = 0
    minimizer: object = None
    stream: object = None
    event: object = None
    out: tuple = field(default_factory=tuple)
    pos_dev: object = None
    t_admit: float = 0.0


def estimate_device_bytes(n_atoms: int, k: int, hist_m: int = 0) -> int:
    """Device bytes one request holds while admitted (tables + coordinates + scratch)."""
    n = 3 * n_atoms
    tables = 64 * n_atoms * 12 + (n_atoms * n_atoms) // 4 + 4096
    coords = 4 * n * k + 16 * k
    mat = (2 * hist_m * n if hist_m else n * n) * 4
    return tables + coords + mat * min(k, 148 * 2) + (1 << 16)


class MMFFServer:
    """Admission-by-budget continuous batching over CUDA streams."""

    def __init__(self, hbm_budget_bytes: int = 8 << 30, n_streams: int = 16, prep_workers: int = 4,
                 device=None, default_max_iters: int = 1000):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("MMFFServer needs a CUDA device")
        self.torch = torch
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.budget = int(hbm_budget_bytes)
        self.in_use = 0
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(n_streams)]
        self.free_streams = list(range(n_streams))
        self.default_max_iters = default_max_iters
        self.pool = ThreadPoolExecutor(max_workers=prep_workers)
        self.incoming: "queue.Queue[_Req]" = queue.Queue()
        self.waiting: list[_Req] = []
        self.running: list[_Req] = []
        self.next_id = 0
        self.lock = threading.Lock()
        self.stop_flag = threading.Event()
        self.peak_in_use = 0
        self.completed = 0
        self.thread = threading.Thread(target=self._loop, name="mmff-server", daemon=True)
        self.thread.start()

    # --- client side ---
    def submit(self, mol, positions: Optional[np.ndarray] = None, variant: str = "MMFF94",
               max_iters: Optional[int] = None) -> Future:
        """Queue one molecule; positions (k, N, 3) default to all of the molecule's conformers."""
        if positions is None:
            positions = np.stack([np.asarray(c.pos if hasattr(c, "pos") else c.GetPositions())
                                  for c in mol.GetConformers()])
        positions = np.asarray(positions, dtype=np.float32).reshape(-1, mol.GetNumAtoms(), 3)
        with self.lock:
            rid = self.next_id
            self.next_id += 1
        fut: Future = Future()
        r = _Req(rid, mol, positions, variant, int(max_iters or self.default_max_iters),
                 time.perf_counter(), fut)
        r.prep = self.pool.submit(self._prepare, r)
        self.incoming.put(r)
        return fut

    def close(self) -> None:
        self.stop_flag.set()
        self.thread.join()
        self.pool.shutdown(wait=True)

    # --- scheduler side ---
    @staticmethod
    def _prepare(r: _Req):
        r.params = extract_mmff_params(r.mol, conf_id=r.mol.GetConformers()[0].GetId()
                                       if r.mol.GetNumConformers() else 0, mmff_variant=r.variant)
        hist = mm.LBFGS_M if r.params.n_atoms >= mm.LBFGS_ATOM_THRESHOLD else 0
        r.nbytes = estimate_device_bytes(r.params.n_atoms, r.positions.shape[0], hist)
        return r

    def _admit(self, r: _Req) -> None:
        torch = self.torch
        sidx = self.free_streams.pop()
        stream = self.streams[sidx]
        r.stream = sidx
        hist = mm.LBFGS_M if r.params.n_atoms >= mm.LBFGS_ATOM_THRESHOLD else 0
        with torch.cuda.stream(stream):
            m = mm.Minimizer([r.params], [r.positions.shape[0]], device=self.device)
            pos = torch.from_numpy(r.positions.reshape(-1).copy()).pin_memory()
            r.pos_dev = pos.to(self.device, non_blocking=True)
            r.out = m.minimize_device(r.pos_dev, max_iters=r.max_iters, history_m=hist, stream=stream)
            r.event = torch.cuda.Event()
            r.event.record(stream)
        r.minimizer = m
        r.t_admit = time.perf_counter()
        self.in_use += r.nbytes
        self.peak_in_use = max(self.peak_in_use, self.in_use)
        self.running.append(r)

    def _finish(self, r: _Req) -> None:
        e, st, it = (t.cpu().numpy() for t in r.out)
        k, n = r.positions.shape[0], r.positions.shape[1]
        pos = r.pos_dev.cpu().numpy().reshape(k, n, 3)
        res = RequestResult(r.rid, pos, e, st, np.isin(st, mm.CONVERGED_STATUSES), r.t_submit, r.t_admit,
                            time.perf_counter())
        self.in_use -= r.nbytes
        self.free_streams.append(r.stream)
        r.minimizer = None
        r.pos_dev = None
        self.completed += 1
        r.future.set_result(res)

    def _loop(self) -> None:
        torch = self.torch
        torch.cuda.set_device(self.device)
        while True:
            try:
                while True:
                    self.waiting.append(self.incoming.get_nowait())
            except queue.Empty:
                pass
            still = []
            for r in self.running:
                if r.event.query():
                    try:
                        self._finish(r)
                    except Exception as exc:  # pragma: no cover - surfaced to the client
                        r.future.set_exception(exc)
                else:
                    still.append(r)
            self.running = still
            keep = []
            for r in self.waiting:
                if not r.prep.done():
                    keep.append(r)
                    continue
                if r.prep.exception() is not None:
                    r.future.set_exception(r.prep.exception())
                    continue
                if r.nbytes > self.budget:
                    r.future.set_exception(MemoryError(
                        f"request {r.rid} needs {r.nbytes} B, above the {self.budget} B budget"))
                    continue
                if self.free_streams and self.in_use + r.nbytes <= self.budget:
                    try:
                        self._admit(r)
                    except Exception as exc:
                        r.future.set_exception(exc)
                else:
                    keep.append(r)
            self.waiting = keep
            if self.stop_flag.is_set() and not self.waiting and not self.running and self.incoming.empty():
                break
            time.sleep(0.0002)


def poisson_stream(server: MMFFServer, make_request, rate_confs_per_s: float, duration_s: float,
                   seed: int = 0):
    """Drive the server with Poisson arrivals; returns the list of futures and submit times."""
    rng = np.random.default_rng(seed)
    futures = []
    t0 = time.perf_counter()
    t_next = t0
    i = 0
    while True:
        mol, positions, variant = make_request(i)
        k = positions.shape[0]
        t_next += rng.exponential(k / rate_confs_per_s)
        now = time.perf_counter()
        if t_next - t0 > duration_s:
            break
        if t_next > now:
            time.sleep(t_next - now)
        futures.append(server.submit(mol, positions, variant))
        i += 1
    return futures
