"""Continuous-batching MMFF optimisation service on one GPU, with slot-level admission.

Requests (one molecule x k conformers, MMFF94 or MMFF94s) arrive at any
time.  The service

* prepares each request on the host in a small thread pool, overlapping the
  GPU: term extraction and native packing of the molecule's device tables,
  cached per molecular graph and MMFF variant (repeat molecules skip both);
* keeps, per size class, a device arena in two halves and a persistent
  worker launch (``mmffb_minimize_queue``) that takes conformer slots from a
  device work queue while it runs.  A prepared request is copied into the
  open half of its class -- tables, slot descriptors, coordinates -- on the
  class's copy stream, followed by the queue's new tail, so the running
  worker's CTAs pick its conformers up as soon as they finish their current
  ones: a request admitted while others are on the GPU joins the running
  launch instead of waiting for the next one;
* learns that a slot is finished from a flag the kernel writes to mapped host
  memory, copies each finished request's results back and completes its
  future.

A worker CTA whose queue stays empty for ``worker_idle_ms`` (1 ms by default)
ends (every wait in the kernel is bounded) and frees its SM for the other
classes.  New slots go first to spare CTAs of a launch younger than that limit
and otherwise start a new launch sized to them; several launches may share a
queue.  A half is filled in order and refilled only when its worker
launches have ended and its requests are complete, so no running launch ever
reads memory written after it started; the other half takes the requests
meanwhile.  Device memory is bounded by the budget: arenas and worker scratch
per size class.

Size classes fix the kernel instance: each class launches with a fixed atom
bound and class-table size, so the instance (CTA size, Hessian in shared
memory or in a global slot, dense BFGS or L-BFGS) depends on the class only.
The kernel's result for a conformer depends only on the instance (slots are
claimed from a queue and no value crosses conformers), so a request's result
is bit-for-bit the same alone or in any mix of requests.

| atoms   | optimizer   | atom bound | class-table bound |
|---------|-------------|------------|-------------------|
| <= 24   | dense BFGS  | 24         | 64                |
| 25-48   | dense BFGS  | 48         | 64                |
| 49-149  | dense BFGS  | 149        | 32                |
| 49-149 with more than 32 non-bonded classes | dense BFGS | 149 | 64 |
| 150-170 | L-BFGS m=8  | 170        | 32                |
| 150-170 with more than 32 non-bonded classes | L-BFGS m=8 | 170 | 64 |
| 171-288 | L-BFGS m=8  | 288        | 32                |
| 171-288 with more than 32 non-bonded classes | L-BFGS m=8 | 288 | 64 |
| 289-400 | L-BFGS m=8  | 400        | 64                |
| > 400   | L-BFGS m=8  | its own    | 64                |

Molecules of 150 atoms or more use L-BFGS, as in the reference pipeline
(mlxmolkit/conformer_pipeline_v2.py:448-452), decided per molecule.  The
150-170 and 171-288-atom L-BFGS classes keep their launch shape small (32
class-table entries) so that their instances fit two CTAs per SM: the
register-capped ones, with the history in shared memory and in a global slot.
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
from .pack import (MD_ATOM_OFF, MD_B_OFF, MD_CLS_OFF, MD_MASK_OFF, MD_NCLS, merge_packed,
                   pack_molecules)


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
        if n_atoms <= 170:
            if n_classes > 32:
                return SizeClass(("lbfgs", 170, 64), 170, 64, mm.LBFGS_M)
            return SizeClass(("lbfgs", 170), 170, 32, mm.LBFGS_M)
        if n_atoms <= 288:
            if n_classes > 32:
                return SizeClass(("lbfgs", 288, 64), 288, 64, mm.LBFGS_M)
            return SizeClass(("lbfgs", 288), 288, 32, mm.LBFGS_M)
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


@dataclass
class _Caps:
    """Capacity of one half of a size class's device arena."""
    slots: int
    coords: int
    mols: int
    rows: int
    atoms: int
    pairs: int
    words: int

    def nbytes(self) -> int:
        return (self.slots * (4 + 8 + 8 + 4 + 4) + self.coords * 4 + self.mols * 64 + self.rows * 16
                + self.atoms * 12 + self.pairs * 8 + self.words * 4 + 16)


def arena_caps(cls: SizeClass, half_bytes: int, max_slots: int = 4096) -> Optional[_Caps]:
    """The largest half arena of class ``cls`` within ``half_bytes`` (None if not even 2 slots fit).

    Tables are provisioned for one molecule per two conformer slots, each molecule at the
    class's atom bound: 40 bonded records and 12 B per atom, the class table and the bit rows.
    """
    n = cls.nmax
    w = (n + 31) // 32

    def caps(slots):
        mols = max(1, slots // 2)
        return _Caps(slots, slots * 3 * n, mols, mols * 40 * n, mols * n, mols * cls.max_classes ** 2,
                     mols * 2 * n * w)
    slots = max_slots
    while slots >= 2 and caps(slots).nbytes() > half_bytes:
        slots //= 2
    return caps(slots) if slots >= 2 else None


class _Half:
    """One half of a size class's device arena: the tables, conformer slots and results of the
    requests one worker generation serves.  Addresses are handed out in order (bump pointers)
    and the half is refilled only after its worker ended, so no running launch reads memory
    written after it started."""

    def __init__(self, srv, caps: _Caps):
        torch = srv.torch
        dev = srv.device
        z = lambda n, dt: torch.zeros(max(int(n), 1), dtype=dt, device=dev)
        self.caps = caps
        self.mol_desc = z(16 * caps.mols, torch.int32)
        self.bonded = z(4 * caps.rows, torch.int32)
        self.atom_cls = z(caps.atoms, torch.int32)
        self.atom_q = z(caps.atoms, torch.float64)
        self.cls_tab = z(2 * caps.pairs, torch.float32)
        self.pair_mask = z(caps.words, torch.int32)
        self.conf_mol = z(caps.slots, torch.int32)
        self.conf_coord = z(caps.slots, torch.int64)
        self.pos = z(caps.coords, torch.float32)
        self.energy = z(caps.slots, torch.float64)
        self.status = z(caps.slots, torch.int32)
        self.iters = z(caps.slots, torch.int32)
        self.ctl = z(4, torch.int32)              # head, tail (published slots), close
        self.done_buf = _lib.MappedHostArray(caps.slots, np.int32)   # per-slot "results written" flags
        self.done_np = self.done_buf.array
        self.done_dev = self.done_buf.device_ptr
        self.workers: list = []                   # (end event, scratch index, launch time) of its launches
        self.pending: list = []                   # queue writes waiting for their data: (event, tail | None)
        self.published = 0                        # the tail written last
        self.closed = True
        self.requests: list = []
        self.n_mol = self.n_row = self.n_atom = self.n_pair = self.n_word = self.n_slot = self.n_coord = 0

    def start(self, stream) -> None:
        """Empty the half for a new generation (no worker of it may be running)."""
        import torch
        self.n_mol = self.n_row = self.n_atom = self.n_pair = self.n_word = self.n_slot = self.n_coord = 0
        self.published = 0
        self.done_np[:] = 0
        with torch.cuda.stream(stream):
            self.ctl.zero_()
        self.closed = False
        self.requests = []

    def fits(self, pk, k: int, n_atoms: int) -> bool:
        return _fits(self, self.caps, pk, k, n_atoms)

    def reserve(self, r) -> None:
        """Hand the request its molecule, records, atoms, class table, bit rows, slots and
        coordinates (in order, so a tick's requests are contiguous)."""
        pk, k, n = r.packed, r.positions.shape[0], int(r.params.n_atoms)
        r.half = self
        r.base = (self.n_mol, self.n_row, self.n_atom, self.n_pair, self.n_word, self.n_slot, self.n_coord)
        r.slot0, r.coord0 = self.n_slot, self.n_coord
        self.n_mol += 1
        self.n_row += len(pk.bonded)
        self.n_atom += len(pk.atom_cls)
        self.n_pair += len(pk.cls_tab)
        self.n_word += len(pk.pair_mask)
        self.n_slot += k
        self.n_coord += 3 * n * k
        self.requests.append(r)

    def live_workers(self) -> list:
        """Launches on this half that have not ended (ended ones are dropped)."""
        self.workers = [w for w in self.workers if not w["ev"].query()]
        return self.workers

    def worker_running(self) -> bool:
        return bool(self.live_workers())

    def idle(self) -> bool:
        """Closed, no worker running and every request completed: free for a new generation."""
        return self.closed and not self.pending and not self.worker_running() and not self.requests


class _ClassState:
    STREAMS = 16                  # concurrent worker launches per class at most

    def __init__(self, srv, key, cls: SizeClass, max_iters: int, caps: _Caps):
        torch = srv.torch
        self.key = key
        self.cls = cls
        self.max_iters = max_iters
        self.halves = [_Half(srv, caps), _Half(srv, caps)]
        self.cur = None
        self.copy_stream = torch.cuda.Stream(device=srv.device)
        self.streams = [torch.cuda.Stream(device=srv.device) for _ in range(self.STREAMS)]
        self.stream_busy = [None] * self.STREAMS       # end event of the launch on each stream
        # the arenas were zeroed on the allocating stream: order every later use after it
        self.copy_stream.wait_stream(torch.cuda.current_stream(srv.device))
        self.opt = mm.opt_params(max_iters, 1e-4, cls.history_m, "mixed")
        bd, cd = self._descs(self.halves[0])
        self.full_grid = int(srv.lib.mmffb_minimize_ctas(ctypes.byref(bd), ctypes.byref(cd), ctypes.byref(self.opt)))
        if self.full_grid <= 0:
            _lib.check(self.full_grid or _lib.MMFFB_EINVAL, "mmffb_minimize_ctas")
        self.slot_scratch = srv.lib.mmffb_queue_scratch_bytes(ctypes.byref(bd), ctypes.byref(cd),
                                                              ctypes.byref(self.opt), 1) - 256
        self.nbytes = 2 * caps.nbytes()
        self.scratch_live: list = []                  # (end event, scratch tensor) of running launches
        self.launches = 0

    def free_stream(self) -> Optional[int]:
        for i, ev in enumerate(self.stream_busy):
            if ev is None or ev.query():
                self.stream_busy[i] = None
                return i
        return None

    def scratch_bytes_live(self) -> int:
        self.scratch_live = [(ev, t) for ev, t in self.scratch_live if not ev.query()]
        return sum(t.numel() for _, t in self.scratch_live)

    def _descs(self, h: _Half):
        c = h.caps
        bd = _lib.MMFFBatchDev(c.mols, self.cls.nmax, self.cls.max_classes, h.mol_desc.data_ptr(),
                               h.bonded.data_ptr(), h.atom_cls.data_ptr(), h.atom_q.data_ptr(),
                               h.cls_tab.data_ptr(), h.pair_mask.data_ptr())
        cd = _lib.MMFFConfDev(c.slots, self.cls.nmax, h.conf_mol.data_ptr(), h.conf_coord.data_ptr(), 0)
        return bd, cd


class MMFFServer:
    """Continuous batching with slot-level admission: one persistent worker per size class takes
    conformer slots from a device work queue while it runs."""

    SLEEP_NS = 20000          # pause between a worker's polls of an empty queue

    def __init__(self, hbm_budget_bytes: int = 8 << 30, prep_workers: int = 4, device=None,
                 default_max_iters: int = 1000, default_max_iters_lbfgs: int = 3000,
                 max_slots_per_half: int = 4096, prep_cache_size: int = 4096, worker_idle_ms: float = 1.0,
                 min_worker_ctas: int = 0):
        """``worker_idle_ms``: a worker CTA whose queue stays empty this long ends.
        ``min_worker_ctas``: launch at least this many CTAs per worker (spare CTAs take slots
        published while they wait)."""
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("MMFFServer needs a CUDA device")
        self.IDLE_POLLS = max(1, int(worker_idle_ms * 1e6 / self.SLEEP_NS))
        self.idle_s = self.IDLE_POLLS * self.SLEEP_NS * 1e-9
        self.min_worker_ctas = int(min_worker_ctas)
        self.torch = torch
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.budget = int(hbm_budget_bytes)
        self.in_use = 0
        self.default_max_iters = default_max_iters
        self.default_max_iters_lbfgs = default_max_iters_lbfgs
        self.max_slots_per_half = int(max_slots_per_half)
        self.pool = ThreadPoolExecutor(max_workers=prep_workers)
        self.incoming: "queue.Queue[_Req]" = queue.Queue()
        self.waiting: list[_Req] = []
        self.copying: list = []               # (request, event, host results)
        self.classes: dict = {}
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
        self.error: Optional[BaseException] = None
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
            packed = _chunk_aligned(pack_molecules([params]))
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
    def _class_state(self, r: _Req) -> Optional[_ClassState]:
        key = (r.cls, r.max_iters)
        cs = self.classes.get(key)
        if cs is None:
            caps = arena_caps(r.cls, max(self.budget // 12, 0), self.max_slots_per_half)
            if caps is None:
                raise MemoryError(f"request {r.rid}: the {self.budget} B budget holds no arena for its size class")
            cs = _ClassState(self, key, r.cls, r.max_iters, caps)
            if self.in_use + cs.nbytes > self.budget:
                raise MemoryError(f"request {r.rid}: size class {r.cls.key} needs {cs.nbytes} B of arenas, "
                                  f"{self.budget - self.in_use} B of the budget are left")
            self.in_use += cs.nbytes
            self.peak_in_use = max(self.peak_in_use, self.in_use)
            self.classes[key] = cs
        return cs

    def _half_for(self, cs: _ClassState, r: _Req, to_close: list) -> Optional[_Half]:
        """The open half that takes r, switching generations when the current one is full (the
        full half is closed after this tick's slots are published)."""
        k, n = r.positions.shape[0], int(r.params.n_atoms)
        if not _fits(_EmptyHalf(), cs.halves[0].caps, r.packed, k, n):
            raise MemoryError(f"request {r.rid} ({k} conformers of {n} atoms) exceeds its size class's arena")
        h = cs.cur
        if h is not None and not h.closed and h.fits(r.packed, k, n):
            return h
        other = cs.halves[1] if h is cs.halves[0] else cs.halves[0]
        if not other.idle():
            return None                       # both halves busy: r waits
        if h is not None and not h.closed:
            h.closed = True
            to_close.append((cs, h))
        other.start(cs.copy_stream)
        cs.cur = other
        return other

    def _close_half(self, cs: _ClassState, h: _Half) -> None:
        """No more slots: the worker ends once it has claimed every published one.  The close flag
        is written after the half's pending tails (in order)."""
        h.pending.append((None, None))
        h.closed = True

    def _flush(self, cs: _ClassState) -> None:
        """Write the queue words whose data has landed, in order: a tail only once the host has
        seen the copies of its slots' data complete, so that a running worker never claims a slot
        before its tables and coordinates are in device memory; the close flag after the tails."""
        torch = self.torch
        for h in cs.halves:
            wrote = 0
            while h.pending:
                ev, tail = h.pending[0]
                if ev is not None and not ev.query():
                    break
                h.pending.pop(0)
                with torch.cuda.stream(cs.copy_stream):
                    if tail is None:
                        h.ctl[2:3].copy_(torch.ones(1, dtype=torch.int32).pin_memory(), non_blocking=True)
                    else:
                        h.ctl[1:2].copy_(torch.tensor([tail], dtype=torch.int32).pin_memory(), non_blocking=True)
                        wrote += tail - h.published
                        h.published = tail
            if wrote:
                ready = torch.cuda.Event()
                ready.record(cs.copy_stream)
                self._ensure_worker(cs, h, ready, wrote)

    def _publish(self, cs: _ClassState, h: _Half, reqs) -> None:
        """Copy the requests' tables, slot descriptors and coordinates into their reserved, contiguous
        places in the half; the new tail follows once they have landed (``_flush``)."""
        torch = self.torch
        pk = merge_packed([r.packed for r in reqs])
        m0, row0, atom0, pair0, word0, slot0, coord0 = reqs[0].base
        desc = pk.mol_desc.copy()
        desc[:, MD_ATOM_OFF] += atom0
        desc[:, MD_CLS_OFF] += pair0
        desc[:, MD_MASK_OFF] += word0
        for t in range(5):
            desc[:, MD_B_OFF + 2 * t] += row0
        counts = [r.positions.shape[0] for r in reqs]
        conf_mol = (np.repeat(np.arange(len(reqs)), counts) + m0).astype(np.int32)
        sizes = np.repeat(3 * pk.n_atoms.astype(np.int64), counts)
        coord = coord0 + np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        pos = np.concatenate([r.positions.reshape(-1) for r in reqs]).astype(np.float32)
        t_admit = time.perf_counter()
        for r in reqs:
            r.t_admit = t_admit

        def put(dst, start, arr, dtype):
            a = torch.from_numpy(np.ascontiguousarray(arr).reshape(-1).view(dtype)).pin_memory()
            dst[start:start + a.numel()].copy_(a, non_blocking=True)

        with torch.cuda.stream(cs.copy_stream):
            put(h.mol_desc, 16 * m0, desc, np.int32)
            put(h.bonded, 4 * row0, pk.bonded, np.int32)
            put(h.atom_cls, atom0, pk.atom_cls, np.int32)
            put(h.atom_q, atom0, pk.atom_q, np.float64)
            put(h.cls_tab, 2 * pair0, pk.cls_tab, np.float32)
            put(h.pair_mask, word0, pk.pair_mask, np.int32)
            put(h.conf_mol, slot0, conf_mol, np.int32)
            put(h.conf_coord, slot0, coord, np.int64)
            put(h.pos, coord0, pos, np.float32)
            landed = torch.cuda.Event()
            landed.record(cs.copy_stream)
        h.pending.append((landed, slot0 + len(conf_mol)))     # the new tail, once the data has landed

    def _ensure_worker(self, cs: _ClassState, h: _Half, ready, new_slots: int) -> None:
        """CTAs for ``new_slots`` just-published slots of h.  Spare CTAs of a launch younger than the
        idle limit are still polling and take them first; the rest get a new launch sized to them
        (at least ``min_worker_ctas``, at most the class's full grid).  Launches share the queue, so
        whichever CTA frees up first takes the next slot."""
        now = time.perf_counter()
        for w in h.live_workers():
            if new_slots <= 0:
                return
            if now - w["t"] < self.idle_s and w["spare"] > 0:
                take = min(w["spare"], new_slots)
                w["spare"] -= take
                new_slots -= take
        if new_slots <= 0:
            return
        i = cs.free_stream()
        if i is None:
            return                          # the running launches take the slots as CTAs free up
        grid = int(min(cs.full_grid, max(new_slots, self.min_worker_ctas)))
        per_cta = max(int(cs.slot_scratch), 0)
        room = max(self.budget - self.in_use - cs.scratch_bytes_live(), 0)
        if per_cta and 256 + grid * per_cta > room:
            grid = int(max(1, min(grid, (room - 256) // per_cta)))
        self._launch_worker(cs, h, ready, i, grid, 256 + grid * per_cta, grid - min(grid, new_slots))

    def _launch_worker(self, cs: _ClassState, h: _Half, ready, i: int, grid: int, scratch_bytes: int,
                       spare: int) -> None:
        torch = self.torch
        L = self.lib
        stream = cs.streams[i]
        stream.wait_event(ready)
        bd, cd = cs._descs(h)
        q = _lib.MMFFQueueDev(h.ctl.data_ptr(), h.ctl.data_ptr() + 4, h.ctl.data_ptr() + 8, h.done_dev,
                              self.IDLE_POLLS, self.SLEEP_NS)
        with torch.cuda.stream(stream):
            sc = torch.empty(scratch_bytes, dtype=torch.uint8, device=self.device)
        rc = L.mmffb_minimize_queue(ctypes.byref(bd), ctypes.byref(cd), ctypes.byref(cs.opt), ctypes.byref(q),
                                    h.pos.data_ptr(), h.energy.data_ptr(), h.status.data_ptr(),
                                    h.iters.data_ptr(), grid, sc.data_ptr(), sc.numel(),
                                    ctypes.c_void_p(stream.cuda_stream))
        _lib.check(rc, "mmffb_minimize_queue")
        ev = torch.cuda.Event()
        ev.record(stream)
        h.workers.append({"ev": ev, "t": time.perf_counter(), "grid": grid, "spare": spare})
        cs.stream_busy[i] = ev
        cs.scratch_live.append((ev, sc))
        cs.launches += 1
        self.launches += 1

    def _collect(self, cs: _ClassState) -> None:
        """Requests whose slots are all done: copy their results back (copy stream)."""
        torch = self.torch
        for h in cs.halves:
            keep = []
            for r in h.requests:
                k, n = r.positions.shape[0], r.positions.shape[1]
                if not h.done_np[r.slot0:r.slot0 + k].all():
                    keep.append(r)
                    continue
                with torch.cuda.stream(cs.copy_stream):
                    hp = torch.empty(3 * n * k, dtype=torch.float32).pin_memory()
                    he = torch.empty(k, dtype=torch.float64).pin_memory()
                    hs = torch.empty(k, dtype=torch.int32).pin_memory()
                    hp.copy_(h.pos[r.coord0:r.coord0 + 3 * n * k], non_blocking=True)
                    he.copy_(h.energy[r.slot0:r.slot0 + k], non_blocking=True)
                    hs.copy_(h.status[r.slot0:r.slot0 + k], non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(cs.copy_stream)
                self.copying.append((r, ev, hp, he, hs))
            h.requests = keep
            # a worker that ended on an empty queue leaves later slots unclaimed: start another
            if keep and not h.pending and not h.worker_running():
                ready = torch.cuda.Event()
                ready.record(cs.copy_stream)
                self._ensure_worker(cs, h, ready, sum(r.positions.shape[0] for r in keep))

    def _finish_copies(self) -> None:
        keep = []
        t = time.perf_counter()
        for item in self.copying:
            r, ev, hp, he, hs = item
            if not ev.query():
                keep.append(item)
                continue
            k, n = r.positions.shape[0], r.positions.shape[1]
            st = hs.numpy().copy()
            r.future.set_result(RequestResult(r.rid, hp.numpy().reshape(k, n, 3).copy(), he.numpy().copy(), st,
                                              np.isin(st, mm.CONVERGED_STATUSES), r.t_submit, r.t_admit, t))
            self.completed += 1
        self.copying = keep

    def _admit(self) -> None:
        """Reserve and publish every prepared request in its size class's open half, in arrival order."""
        keep = []
        groups: dict = {}
        to_close: list = []
        for r in self.waiting:
            if not r.prep.done():
                keep.append(r)
                continue
            if r.prep.exception() is not None:
                r.future.set_exception(r.prep.exception())
                continue
            try:
                cs = self._class_state(r)
                h = self._half_for(cs, r, to_close)
            except MemoryError as exc:
                r.future.set_exception(exc)
                continue
            if h is None:
                keep.append(r)
                continue
            h.reserve(r)
            groups.setdefault((id(cs), id(h)), (cs, h, []))[2].append(r)
        for cs, h, reqs in groups.values():
            try:
                self._publish(cs, h, reqs)
            except Exception as exc:        # pragma: no cover - surfaced to the clients
                for r in reqs:
                    if not r.future.done():
                        r.future.set_exception(exc)
                h.requests = [x for x in h.requests if x not in reqs]
        for cs, h in to_close:
            self._close_half(cs, h)
        self.waiting = keep

    def _fail_all(self, exc: BaseException) -> None:
        """Complete every request not yet completed with ``exc``: waiting, published, copying."""
        open_reqs = list(self.waiting) + [item[0] for item in self.copying]
        for cs in self.classes.values():
            for h in cs.halves:
                open_reqs += h.requests
                h.requests = []
        for r in open_reqs:
            if not r.future.done():
                r.future.set_exception(exc)
        self.waiting = []
        self.copying = []

    def _loop(self) -> None:
        torch = self.torch
        torch.cuda.set_device(self.device)
        while True:
            try:
                while True:
                    self.waiting.append(self.incoming.get_nowait())
            except queue.Empty:
                pass
            try:
                for cs in list(self.classes.values()):
                    self._flush(cs)
                    self._collect(cs)
                self._finish_copies()
                self._admit()
            except BaseException as exc:    # pragma: no cover - fail every open request with it
                import sys
                import traceback
                traceback.print_exc(file=sys.stderr)
                self.error = exc
                self._fail_all(exc)
            pending = any(h.requests or h.pending for cs in self.classes.values() for h in cs.halves)
            if self.stop_flag.is_set() and not self.waiting and not pending and not self.copying \
                    and self.incoming.empty():
                for cs in self.classes.values():
                    for h in cs.halves:
                        if not h.closed:
                            self._close_half(cs, h)
                    self._flush(cs)
                for cs in self.classes.values():
                    cs.copy_stream.synchronize()
                    for st in cs.streams:
                        st.synchronize()
                break
            time.sleep(0.0002)


class _EmptyHalf:
    """Counters of an empty half (the capacity check of a request alone)."""

    n_mol = n_row = n_atom = n_pair = n_word = n_slot = n_coord = 0


def _chunk_aligned(pk):
    """The molecule's bonded records padded to whole chunks of 32 (512 bytes): a molecule without
    bonded terms packs as one invalid record, and every molecule's records must start on a
    512-byte boundary of the arena (a worker keeps them in its read-only cache)."""
    rows = len(pk.bonded)
    if rows % 32 == 0:
        return pk
    pad = np.zeros((32 - rows % 32, 4), dtype=np.uint32)
    pad[:, 0] = 0xFFFFFFFF
    pk.bonded = np.concatenate([pk.bonded, pad])
    return pk


def _fits(h, c: _Caps, pk, k: int, n_atoms: int) -> bool:
    """Whether one more molecule (packed tables pk) with k conformers fits after h's counters."""
    return (h.n_mol + 1 <= c.mols and h.n_row + len(pk.bonded) <= c.rows
            and h.n_atom + len(pk.atom_cls) <= c.atoms and h.n_pair + len(pk.cls_tab) <= c.pairs
            and h.n_word + len(pk.pair_mask) <= c.words and h.n_slot + k <= c.slots
            and h.n_coord + 3 * n_atoms * k <= c.coords)


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
