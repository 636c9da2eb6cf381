"""Continuous-batching MMFF optimisation service on one GPU.

Requests (one molecule x k conformers, MMFF94 or MMFF94s) arrive at any
time.  The service

* prepares each request on the host in a small thread pool, overlapping the
  GPU: term extraction and packing of the molecule's device tables, cached
  per molecular graph and MMFF variant (repeat molecules skip both);
* sorts prepared requests into size classes (below).  Whenever a CUDA stream
  is free and the device-memory budget allows, it launches all the waiting
  requests of a class, up to a conformer cap, as ONE persistent optimizer
  launch.  Requests that arrive while others are on the GPU therefore join
  the next launch of their class, and launches of different classes and
  successive launches overlap on separate streams;
* keeps a launch's coordinates, tables, optimizer scratch and results
  resident on the device until the kernel ends.  The tables, coordinates and
  results go through pinned staging buffers owned by the stream and reused
  from launch to launch.  The service then completes each request's future.

Size classes fix the kernel instance: each class launches with a fixed atom
bound and class-table size, so the instance (CTA size, Hessian in shared
memory or in a global slot, dense BFGS or L-BFGS) depends on the class only.
The kernel's result for a conformer depends only on the instance (work is
pulled from a queue and no value crosses conformers), so a request's result
is bit-for-bit the same alone or in any mix of requests.

| atoms   | optimizer   | atom bound | class-table bound |
|---------|-------------|------------|-------------------|
| <= 24   | dense BFGS  | 24         | 64                |
| 25-48   | dense BFGS  | 48         | 64                |
| 49-149  | dense BFGS  | 149        | 32                |
| 49-149 with more than 32 non-bonded classes | dense BFGS | 149 | 64 |
| 150-300 | L-BFGS m=8  | 300        | 64                |
| 301-400 | L-BFGS m=8  | 400        | 64                |
| > 400   | L-BFGS m=8  | its own    | 64                |

Molecules of 150 atoms or more use L-BFGS, as in the reference pipeline
(mlxmolkit/conformer_pipeline_v2.py:448-452), decided per molecule.
"""
from __future__ import annotations

import ctypes
import queue
from collections import OrderedDict
import threading
import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from . import mmff_minimize as mm
from .mmff_params import extract_mmff_params
from .pack import MD_NCLS, conformer_index, lpt_order, merge_packed, pack_molecules


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


@dataclass(frozen=True)
class SizeClass:
    key: tuple
    nmax: int          # atom bound of the launch
    max_classes: int   # class-table bound of the launch
    history_m: int     # 0: dense BFGS


def size_class(n_atoms: int, n_classes: int) -> SizeClass:
    """The launch class of a molecule (a function of its own atom and class counts)."""
    if n_atoms >= mm.LBFGS_ATOM_THRESHOLD:
        if n_atoms <= 300:
            return SizeClass(("lbfgs", 300), 300, 64, mm.LBFGS_M)
        if n_atoms <= 400:
            return SizeClass(("lbfgs", 400), 400, 64, mm.LBFGS_M)
        return SizeClass(("lbfgs", n_atoms), n_atoms, 64, mm.LBFGS_M)
    if n_atoms <= 24:
        return SizeClass(("dense", 24), 24, 64, 0)
    if n_atoms <= 48:
        return SizeClass(("dense", 48), 48, 64, 0)
    if n_classes > 32:
        return SizeClass(("dense", 149, 64), 149, 64, 0)
    return SizeClass(("dense", 149), 149, 32, 0)


def estimate_device_bytes(n_atoms: int, k: int, hist_m: int = 0) -> int:
    """Device bytes one request's tables, coordinates and results hold while it runs."""
    n = 3 * n_atoms
    tables = 64 * n_atoms * 12 + (n_atoms * n_atoms) // 4 + 4096
    coords = 4 * n * k + 16 * k
    return tables + coords + (1 << 12)


def launch_scratch_bytes(cls: SizeClass, n_conf: int, ctas: int = 2 * 148) -> int:
    """Upper bound of one launch's optimizer scratch: an inverse-Hessian (or history) slot per CTA."""
    n = 3 * cls.nmax
    nv = (n + 3) & ~3
    slot = 2 * cls.history_m * nv if cls.history_m else n * nv
    return 256 + 8 * slot * min(n_conf, ctas)


@dataclass
class _Req:
    rid: int
    mol: object
    positions: np.ndarray          # (k, N, 3) float32
    variant: str
    max_iters: int
    t_submit: float
    future: Future
    prep: Optional[Future] = None
    params: object = None
    packed: object = None
    cls: Optional[SizeClass] = None
    nbytes: int = 0
    t_admit: float = 0.0


# extraction drops non-bonded pairs farther apart than this in the conformer it reads
# (extract_mmff_params' non_bonded_thresh default)
_PAIR_THRESHOLD = 100.0


def _within_pair_threshold(positions: np.ndarray) -> bool:
    """True when no two atoms of the request's first conformer can be farther apart than the
    extraction's pair threshold (bounding-box diagonal), so its tables depend on topology only."""
    p = np.asarray(positions[0], dtype=np.float64)
    return bool(np.linalg.norm(p.max(axis=0) - p.min(axis=0)) <= _PAIR_THRESHOLD)


def topology_key(mol, variant: str):
    """Index-ordered molecular graph: elements, aromaticity, formal charges and bond orders.

    MMFF atom types, charges and every term follow from it, so two requests with the same
    key (and conformers inside the pair threshold) share their device tables.
    """
    atoms = tuple((a.GetSymbol(), bool(a.GetIsAromatic()),
                   int(a.GetFormalCharge()) if hasattr(a, "GetFormalCharge") else 0) for a in mol.GetAtoms())
    bonds = tuple(sorted((min(b.GetBeginAtomIdx(), b.GetEndAtomIdx()), max(b.GetBeginAtomIdx(), b.GetEndAtomIdx()),
                          float(b.GetBondTypeAsDouble())) for b in mol.GetBonds()))
    types = tuple(getattr(mol, "types", None) or ())      # explicit atom types, where the molecule carries them
    return (variant, atoms, bonds, types)


class _Staging:
    """Pinned host and device byte buffers of one stream, grown on demand and reused."""

    def __init__(self, torch, device):
        self.torch = torch
        self.device = device
        self.host: dict = {}
        self.dev: dict = {}

    def _get(self, store, name, nbytes, pinned):
        torch = self.torch
        b = store.get(name)
        if b is None or b.numel() < nbytes:
            size = max(2 * nbytes, 1 << 16)
            b = (torch.empty(size, dtype=torch.uint8, pin_memory=True) if pinned else
                 torch.empty(size, dtype=torch.uint8, device=self.device))
            store[name] = b
        return b

    def upload(self, name, arr: np.ndarray, stream):
        """Copy a host array into this stream's device buffer `name` (async, through pinned memory)."""
        a = np.ascontiguousarray(arr)
        nb = max(a.nbytes, 16)
        h = self._get(self.host, name, nb, True)
        h.numpy()[:a.nbytes] = a.reshape(-1).view(np.uint8)
        d = self._get(self.dev, name, nb, False)
        with self.torch.cuda.stream(stream):
            d[:a.nbytes].copy_(h[:a.nbytes], non_blocking=True)
        return d

    def device_buf(self, name, nbytes):
        return self._get(self.dev, name, max(nbytes, 16), False)

    def download(self, name, dev_buf, nbytes, stream):
        """Queue a device -> pinned host copy; returns the host buffer (valid after the stream syncs)."""
        h = self._get(self.host, name, max(nbytes, 16), True)
        with self.torch.cuda.stream(stream):
            h[:nbytes].copy_(dev_buf[:nbytes], non_blocking=True)
        return h


class _Launch:
    def __init__(self, reqs, cls, stream_idx, event, out, nbytes):
        self.reqs = reqs
        self.cls = cls
        self.stream_idx = stream_idx
        self.event = event
        self.out = out             # (pos host, E host, status host, iters host, offsets)
        self.nbytes = nbytes


class MMFFServer:
    """Admission-by-budget continuous batching: one launch per size class and free stream."""

    def __init__(self, hbm_budget_bytes: int = 8 << 30, n_streams: int = 8, prep_workers: int = 4,
                 device=None, default_max_iters: int = 1000, default_max_iters_lbfgs: int = 3000,
                 max_launch_conformers: int = 4096,
                 prep_cache_size: int = 4096):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("MMFFServer needs a CUDA device")
        self.torch = torch
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.budget = int(hbm_budget_bytes)
        self.in_use = 0
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(n_streams)]
        self.staging = [_Staging(torch, self.device) for _ in range(n_streams)]
        self.free_streams = list(range(n_streams))
        self.default_max_iters = default_max_iters
        self.default_max_iters_lbfgs = default_max_iters_lbfgs
        self.max_launch_conformers = int(max_launch_conformers)
        self.pool = ThreadPoolExecutor(max_workers=prep_workers)
        self.incoming: "queue.Queue[_Req]" = queue.Queue()
        self.waiting: list[_Req] = []
        self.running: list[_Launch] = []
        self.next_id = 0
        self.lock = threading.Lock()
        self.stop_flag = threading.Event()
        self.peak_in_use = 0
        self.completed = 0
        self.launches = 0
        self.prep_cache: "OrderedDict" = OrderedDict()
        self.prep_cache_size = int(prep_cache_size)
        self.prep_hits = 0
        self.lib = _lib.load()
        self.thread = threading.Thread(target=self._loop, name="mmff-server", daemon=True)
        self.thread.start()

    # --- client side ---
    def submit(self, mol, positions: Optional[np.ndarray] = None, variant: str = "MMFF94",
               max_iters: Optional[int] = None) -> Future:
        """Queue one molecule; positions (k, N, 3) default to all of the molecule's conformers.

        ``max_iters`` defaults to ``default_max_iters`` for dense BFGS (below 150 atoms) and
        ``default_max_iters_lbfgs`` for L-BFGS.
        """
        if positions is None:
            positions = np.stack([np.asarray(c.pos if hasattr(c, "pos") else c.GetPositions())
                                  for c in mol.GetConformers()])
        positions = np.asarray(positions, dtype=np.float32).reshape(-1, mol.GetNumAtoms(), 3)
        with self.lock:
            rid = self.next_id
            self.next_id += 1
        fut: Future = Future()
        r = _Req(rid, mol, positions, variant, int(max_iters or 0), time.perf_counter(), fut)
        r.prep = self.pool.submit(self._prepare, r)
        self.incoming.put(r)
        return fut

    def close(self) -> None:
        self.stop_flag.set()
        self.thread.join()
        self.pool.shutdown(wait=True)

    # --- host preparation (thread pool) ---
    def _prepare(self, r: _Req):
        key = topology_key(r.mol, r.variant) if _within_pair_threshold(r.positions) else None
        hit = None
        if key is not None:
            with self.lock:
                hit = self.prep_cache.get(key)
                if hit is not None:
                    self.prep_cache.move_to_end(key)
        if hit is None:
            params = extract_mmff_params(r.mol, conf_id=r.mol.GetConformers()[0].GetId()
                                         if r.mol.GetNumConformers() else 0, mmff_variant=r.variant)
            packed = pack_molecules([params])
            hit = (params, packed, size_class(int(params.n_atoms), int(packed.mol_desc[0, MD_NCLS])))
            if key is not None:
                with self.lock:
                    self.prep_cache[key] = hit
                    while len(self.prep_cache) > self.prep_cache_size:
                        self.prep_cache.popitem(last=False)
        else:
            self.prep_hits += 1
        r.params, r.packed, r.cls = hit
        if r.max_iters <= 0:
            r.max_iters = self.default_max_iters_lbfgs if r.cls.history_m else self.default_max_iters
        r.nbytes = estimate_device_bytes(r.params.n_atoms, r.positions.shape[0], r.cls.history_m)
        return r

    # --- scheduler side ---
    def _launch(self, reqs, cls: SizeClass, sidx: int, nbytes: int) -> None:
        torch = self.torch
        L = self.lib
        stream = self.streams[sidx]
        stg = self.staging[sidx]
        pk = merge_packed([r.packed for r in reqs])
        counts = [r.positions.shape[0] for r in reqs]
        n_atoms = pk.n_atoms.astype(np.int64)
        conf_mol, coord, total = conformer_index(n_atoms, counts)
        order = lpt_order(n_atoms, conf_mol)
        pos = np.concatenate([r.positions.reshape(-1) for r in reqs]).astype(np.float32)
        C = len(conf_mol)
        d_desc = stg.upload("mol_desc", pk.mol_desc.reshape(-1), stream)
        d_bond = stg.upload("bonded", pk.bonded.reshape(-1), stream)
        d_cls = stg.upload("atom_cls", pk.atom_cls, stream)
        d_q = stg.upload("atom_q", pk.atom_q, stream)
        d_tab = stg.upload("cls_tab", pk.cls_tab.reshape(-1), stream)
        d_mask = stg.upload("pair_mask", pk.pair_mask, stream)
        d_cm = stg.upload("conf_mol", conf_mol.astype(np.int32), stream)
        d_co = stg.upload("conf_coord", coord.astype(np.int64), stream)
        d_or = stg.upload("order", order.astype(np.int32), stream)
        d_pos = stg.upload("pos", pos, stream)
        d_e = stg.device_buf("energy", 8 * C)
        d_st = stg.device_buf("status", 4 * C)
        d_it = stg.device_buf("iters", 4 * C)
        bd = _lib.MMFFBatchDev(pk.n_mols, cls.nmax, cls.max_classes, d_desc.data_ptr(), d_bond.data_ptr(),
                               d_cls.data_ptr(), d_q.data_ptr(), d_tab.data_ptr(), d_mask.data_ptr())
        cd = _lib.MMFFConfDev(C, cls.nmax, d_cm.data_ptr(), d_co.data_ptr(), d_or.data_ptr())
        o = mm.opt_params(reqs[0].max_iters, 1e-4, cls.history_m, "mixed")
        need = L.mmffb_minimize_scratch_bytes(ctypes.byref(bd), ctypes.byref(cd), ctypes.byref(o))
        if need == 0:
            _lib.check(_lib.MMFFB_EINVAL, "mmffb_minimize_scratch_bytes")
        scratch = stg.device_buf("scratch", need)
        rc = L.mmffb_minimize(ctypes.byref(bd), ctypes.byref(cd), ctypes.byref(o), d_pos.data_ptr(),
                              d_e.data_ptr(), d_st.data_ptr(), d_it.data_ptr(), None, scratch.data_ptr(),
                              scratch.numel(), ctypes.c_void_p(stream.cuda_stream))
        _lib.check(rc, "mmffb_minimize")
        h_pos = stg.download("pos_out", d_pos, 4 * total, stream)
        h_e = stg.download("energy_out", d_e, 8 * C, stream)
        h_st = stg.download("status_out", d_st, 4 * C, stream)
        h_it = stg.download("iters_out", d_it, 4 * C, stream)
        ev = torch.cuda.Event()
        ev.record(stream)
        t = time.perf_counter()
        for r in reqs:
            r.t_admit = t
        starts = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        self.running.append(_Launch(reqs, cls, sidx, ev, (h_pos, h_e, h_st, h_it, starts, coord, C, total),
                                    nbytes))
        self.in_use += nbytes
        self.peak_in_use = max(self.peak_in_use, self.in_use)
        self.launches += 1

    def _finish(self, ln: _Launch) -> None:
        h_pos, h_e, h_st, h_it, starts, coord, C, total = ln.out
        pos = np.frombuffer(h_pos.numpy(), dtype=np.float32, count=total)
        e = np.frombuffer(h_e.numpy(), dtype=np.float64, count=C)
        st = np.frombuffer(h_st.numpy(), dtype=np.int32, count=C)
        t = time.perf_counter()
        for i, r in enumerate(ln.reqs):
            a, b = int(starts[i]), int(starts[i + 1])
            k, n = r.positions.shape[0], r.positions.shape[1]
            p = pos[int(coord[a]): int(coord[a]) + 3 * n * k].reshape(k, n, 3).copy()
            s = st[a:b].copy()
            r.future.set_result(RequestResult(r.rid, p, e[a:b].copy(), s, np.isin(s, mm.CONVERGED_STATUSES),
                                              r.t_submit, r.t_admit, t))
            self.completed += 1
        self.in_use -= ln.nbytes
        self.free_streams.append(ln.stream_idx)

    def _admit(self) -> None:
        """Launch the waiting, prepared requests of each size class while streams and budget allow."""
        ready: dict = {}
        keep = []
        for r in self.waiting:
            if not r.prep.done():
                keep.append(r)
                continue
            if r.prep.exception() is not None:
                r.future.set_exception(r.prep.exception())
                continue
            alone = r.nbytes + launch_scratch_bytes(r.cls, r.positions.shape[0])
            if alone > self.budget:
                r.future.set_exception(MemoryError(
                    f"request {r.rid} needs {alone} B, above the {self.budget} B budget"))
                continue
            ready.setdefault((r.cls, r.max_iters), []).append(r)
        # oldest request first across classes
        for (cls, _), reqs in sorted(ready.items(), key=lambda kv: kv[1][0].t_submit):
            while reqs and self.free_streams:
                take, confs, nbytes = [], 0, 0
                for r in reqs:
                    k = r.positions.shape[0]
                    if take and confs + k > self.max_launch_conformers:
                        break
                    extra = nbytes + r.nbytes + launch_scratch_bytes(cls, confs + k)
                    if self.in_use + extra > self.budget:
                        break
                    take.append(r)
                    confs += k
                    nbytes += r.nbytes
                if not take:
                    break
                total = nbytes + launch_scratch_bytes(cls, confs)
                sidx = self.free_streams.pop()
                try:
                    self._launch(take, cls, sidx, total)
                except Exception as exc:
                    self.free_streams.append(sidx)
                    for r in take:
                        r.future.set_exception(exc)
                reqs = reqs[len(take):]
            keep.extend(reqs)
        self.waiting = keep

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
            for ln in self.running:
                if ln.event.query():
                    try:
                        self._finish(ln)
                    except Exception as exc:  # pragma: no cover - surfaced to the clients
                        for r in ln.reqs:
                            if not r.future.done():
                                r.future.set_exception(exc)
                else:
                    still.append(ln)
            self.running = still
            self._admit()
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
