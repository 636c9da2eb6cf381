"""Batched MMFF94/94s minimisation on B200 -- the ``mmff_minimize_nk`` drop-in.

Host side of the C ABI in include/mmffb200.h: term tables are packed once per
molecule (``pack.py``), uploaded with PyTorch (device memory, streams), and
the sm_100a kernels of libmmffb200.so do the work.  Nothing here computes
energies on the CPU; without the library or a CUDA device the calls raise.

Reference counterparts:
  mmff_minimize_nk          mlxmolkit/mmff_minimize.py:231-346
  optimizer constants       mlxmolkit/mmff_bfgs_header.metal:3-12
  status -> converged       mlxmolkit/mmff_minimize.py:346 (status == 0)
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from .pack import PackedBatch, conformer_index, lpt_order, pack_molecules

# Optimizer constants TOLX FUNCTOL MOVETOL EPS MAX_STEP_FACTOR MAX_LS GRAD_SCALE GRAD_CAP:
# the reference in-kernel optimizer's (mmff_bfgs_header.metal:3-12) and RDKit's / nvMolKit's
# (mlxmolkit/bfgs_metal.py:23-28).
TG_CONSTS = (1.2e-6, 1e-4, 1e-6, 3e-7, 100.0, 1000.0, 0.1, 10.0)
RDKIT_CONSTS = (1.2e-7, 1e-4, 1e-7, 3e-8, 100.0, 100.0, 0.1, 10.0)
# Term constants {cb, angle/oop prefactor, stretch-bend gradient prefactor, honour linear}:
# in-kernel optimizer header (mmff_bfgs_header.metal:85-87,154,192) and mega/fused kernels
# (mmff_metal_kernel.py:274-280).
MODE_TG = (-0.4 * math.pi / 180.0, 143.9325 * (math.pi / 180.0) ** 2, 143.9325 * math.pi / 180.0, 1.0)
MODE_MEGA = (-0.007, 0.043844, 2.51210, 0.0)
LBFGS_M = 8                    # mlxmolkit/mmff_minimize.py:31
LBFGS_ATOM_THRESHOLD = 150     # mlxmolkit/conformer_pipeline_v2.py:448

CONVERGED_STATUSES = (_lib.ST_GRAD, _lib.ST_TOLX, _lib.ST_SLOPE, _lib.ST_LSFAIL)


def load_tuning(path: Optional[str] = None) -> dict:
    """Per-bin launch configuration written by autotune.py (empty if none)."""
    import json
    import os
    path = path or os.environ.get("MMFFB_TUNING") or os.path.join(os.path.dirname(__file__), "tuning.json")
    try:
        with open(path) as f:
            return json.load(f).get("bins", {})
    except (OSError, ValueError):
        return {}


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise _lib.MMFFBError("no CUDA device: the MMFF kernels run on the GPU only")
    return torch


class DeviceBatch:
    """Packed molecule tables resident in device memory (one upload, many launches)."""

    def __init__(self, packed: PackedBatch, device=None):
        torch = _torch()
        self.packed = packed
        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev, non_blocking=False)
        self.mol_desc = t(packed.mol_desc.reshape(-1))
        self.bonded = t(packed.bonded.view(np.int32).reshape(-1))
        self.atom_cls = t(packed.atom_cls if len(packed.atom_cls) else np.zeros(1, np.int32))
        self.atom_q = t(packed.atom_q if len(packed.atom_q) else np.zeros(1, np.float64))
        self.cls_tab = t(packed.cls_tab.reshape(-1))
        self.pair_mask = t(packed.pair_mask.view(np.int32))
        self.n_atoms = packed.n_atoms
        self.nbytes = sum(x.numel() * x.element_size() for x in (self.mol_desc, self.bonded, self.atom_cls,
                                                                  self.atom_q, self.cls_tab, self.pair_mask))

    @classmethod
    def from_params(cls, params_list, device=None) -> "DeviceBatch":
        return cls(pack_molecules(params_list), device)

    def desc(self) -> _lib.MMFFBatchDev:
        return _lib.MMFFBatchDev(self.packed.n_mols, self.packed.max_atoms, self.packed.max_classes,
                                 self.mol_desc.data_ptr(),
                                 self.bonded.data_ptr(), self.atom_cls.data_ptr(), self.atom_q.data_ptr(),
                                 self.cls_tab.data_ptr(), self.pair_mask.data_ptr())


class DeviceConformers:
    """Conformer -> molecule map, coordinate offsets and processing order on the device."""

    def __init__(self, batch: DeviceBatch, conf_mol: np.ndarray, conf_coord: np.ndarray,
                 order: Optional[np.ndarray] = None):
        torch = _torch()
        dev = batch.device
        self.n_conf = int(len(conf_mol))
        self.conf_mol_np = np.asarray(conf_mol, dtype=np.int32)
        self.max_atoms = int(batch.n_atoms[self.conf_mol_np].max()) if self.n_conf else 1
        self.conf_mol = torch.from_numpy(self.conf_mol_np.copy()).to(dev)
        self.conf_coord = torch.from_numpy(np.asarray(conf_coord, dtype=np.int64).copy()).to(dev)
        self.order = None if order is None else torch.from_numpy(np.asarray(order, np.int32).copy()).to(dev)
        self.nbytes = 12 * self.n_conf + (0 if order is None else 4 * len(order))

    def desc(self) -> _lib.MMFFConfDev:
        return _lib.MMFFConfDev(self.n_conf, self.max_atoms, self.conf_mol.data_ptr(),
                                self.conf_coord.data_ptr(), 0 if self.order is None else self.order.data_ptr())


def opt_params(max_iters: int, grad_tol: float, history_m: int = 0, precision: str = "mixed",
               consts=TG_CONSTS, mode=MODE_TG, threads: int = 0, ctas_per_sm: int = 0,
               exit_test: int = _lib.EXIT_TG, check_every: int = 0,
               atom_grad_scale: float = 1.0, max_restarts: int = 0,
               polish64: Optional[bool] = None, hpass_lean: bool = True, wait_spins: int = 0,
               err_word: int = 0, give_up_waits: bool = False) -> _lib.MMFFOptParams:
    """Launch options.

    ``polish64`` switches a conformer's line-search energies to FP64 once the FP32 ones stall.
    Its default follows the optimizer: off for dense BFGS, whose mixed form is then FP32 terms,
    gradients and update with FP64 only in the energy sums, the Armijo tests and the
    convergence tests; on for mixed-precision L-BFGS, which on flexible 150-400-atom molecules
    otherwise ends most conformers on an FP32 line-search stall short of the minimum.
    ``err_word``: device address of an int32 that the launch sets to 1 when a bounded wait gives
    up; ``wait_spins`` bounds those waits (0: the library default); ``give_up_waits`` makes every
    such wait give up at once (a test switch that exercises the timeout path)."""
    o = _lib.MMFFOptParams()
    o.wait_spins = int(wait_spins)
    o.give_up_waits = int(bool(give_up_waits))
    o.err_word = int(err_word) or None
    o.max_restarts = int(max_restarts)
    o.polish64 = int(precision == "mixed" and history_m > 0 if polish64 is None else bool(polish64))
    o.hpass_lean = int(bool(hpass_lean))
    o.exit_test = int(exit_test)
    o.check_every = int(check_every)
    o.atom_grad_scale = float(atom_grad_scale)
    o.max_iters = int(max_iters)
    o.history_m = int(history_m)
    o.precision = _lib.PREC[precision]
    o.threads = int(threads)
    o.ctas_per_sm = int(ctas_per_sm)
    o.grad_tol = float(grad_tol)
    for i, v in enumerate(consts):
        o.consts[i] = float(v)
    for i, v in enumerate(mode):
        o.mode[i] = float(v)
    return o


def _stream_ptr(torch, stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


@dataclass
class MinimizeResult:
    positions: np.ndarray      # float32, flat, molecule-major conformer order
    energies: np.ndarray       # float64 (C,)
    status: np.ndarray         # int32 (C,) MMFFB_ST_*
    iters: np.ndarray          # int32 (C,)
    # FP64 check at the returned coordinates (mmffb_fp64_check): the FP64 energy, the
    # returned energy's error against it, and the RMS of the FP64 gradient (kcal/mol/A)
    energies_fp64: Optional[np.ndarray] = None
    energy_errors: Optional[np.ndarray] = None
    grad_rms_fp64: Optional[np.ndarray] = None
    timings: Optional[dict] = None     # host seconds of the drop-in call's steps (mmff_minimize_nk)

    @property
    def converged(self) -> np.ndarray:
        return np.isin(self.status, CONVERGED_STATUSES)


class Minimizer:
    """Device-resident minimisation of one packed batch (tables uploaded once)."""

    def __init__(self, params_list, conf_counts: Sequence[int], device=None, packed: Optional[PackedBatch] = None):
        """``packed``: the molecules' tables when already packed (e.g. merged from per-molecule
        packs); ``params_list`` may then be None, the atom counts coming from the tables."""
        if params_list is None and packed is None:
            raise ValueError("give the molecules' parameters or their packed tables")
        self.params_list = list(params_list) if params_list is not None else None
        self.conf_counts = [int(k) for k in conf_counts]
        t = time.perf_counter()
        if packed is None:
            packed = pack_molecules(self.params_list)
            self.pack_s = time.perf_counter() - t
        else:
            self.pack_s = 0.0
        self.batch = DeviceBatch(packed, device)
        n_atoms = [int(v) for v in packed.n_atoms]
        self.conf_mol, self.conf_coord, self.total = conformer_index(n_atoms, self.conf_counts)
        self.order = lpt_order(n_atoms, self.conf_mol)
        self.confs = DeviceConformers(self.batch, self.conf_mol, self.conf_coord, self.order)
        self._scratch = None
        # host -> device bytes of the set-up (tables and conformer index arrays)
        self.upload_bytes = self.batch.nbytes + self.confs.nbytes

    def _scratch_for(self, nbytes: int):
        torch = _torch()
        if self._scratch is None or self._scratch.numel() < nbytes:
            self._scratch = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.batch.device)
        return self._scratch

    def minimize_device(self, pos_dev, *, max_iters: int, grad_tol: float = 1e-4, history_m: int = 0,
                        precision: str = "mixed", consts=TG_CONSTS, mode=MODE_TG, threads: int = 0,
                        ctas_per_sm: int = 0, exit_test: int = _lib.EXIT_TG, check_every: int = 0,
                        atom_grad_scale: float = 1.0, max_restarts: int = 0, polish64=None,
                        hpass_lean: bool = True, stream=None, out=None, evals=None, err=None,
                        wait_spins: int = 0, give_up_waits: bool = False):
        """Minimise in place on the device; returns (energy, status, iters) device tensors.

        ``evals`` (optional int32 device tensor, one per conformer) receives the
        number of energy-only line-search evaluations; ``err`` (optional int32
        device tensor of one element) is set to 1 if a bounded wait inside the
        kernel gave up (its conformers then have status ``ST_TIMEOUT``).
        """
        torch = _torch()
        L = _lib.load()
        C = self.confs.n_conf
        if out is None:
            e = torch.empty(C, dtype=torch.float64, device=self.batch.device)
            st = torch.empty(C, dtype=torch.int32, device=self.batch.device)
            it = torch.empty(C, dtype=torch.int32, device=self.batch.device)
        else:
            e, st, it = out
        o = opt_params(max_iters, grad_tol, history_m, precision, consts, mode, threads, ctas_per_sm,
                       exit_test, check_every, atom_grad_scale, max_restarts, polish64, hpass_lean,
                       wait_spins, err.data_ptr() if err is not None else 0, give_up_waits)
        bd, cd = self.batch.desc(), self.confs.desc()
        nbytes = L.mmffb_minimize_scratch_bytes(ctypes.byref(bd), ctypes.byref(cd), ctypes.byref(o))
        if nbytes == 0 and C > 0:
            _lib.check(-1 if not L.mmffb_last_error() else _lib.MMFFB_EINVAL, "mmffb_minimize_scratch_bytes")
        scratch = self._scratch_for(nbytes)
        rc = L.mmffb_minimize(ctypes.byref(bd), ctypes.byref(cd), ctypes.byref(o), pos_dev.data_ptr(),
                              e.data_ptr(), st.data_ptr(), it.data_ptr(),
                              evals.data_ptr() if evals is not None else None, scratch.data_ptr(),
                              scratch.numel(), _stream_ptr(torch, stream))
        _lib.check(rc, "mmffb_minimize")
        return e, st, it

    def minimize(self, positions: np.ndarray, **kw) -> MinimizeResult:
        """Host-synchronous minimisation; raises ``MMFFBError`` if a bounded wait inside the
        kernel gave up (a result that is not valid, never expected)."""
        torch = _torch()
        pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
        if pos.size != self.total:
            raise ValueError(f"positions hold {pos.size} floats, the conformers need {self.total}")
        pos_dev = torch.from_numpy(pos.copy()).to(self.batch.device)
        err = torch.zeros(1, dtype=torch.int32, device=self.batch.device)
        e, st, it = self.minimize_device(pos_dev, err=err, **kw)
        e64, de, gr = self.fp64_check_device(pos_dev, e, mode=kw.get("mode", MODE_TG))
        torch.cuda.synchronize()
        if int(err.item()):
            raise _lib.MMFFBError("mmffb_minimize: a bounded wait inside the kernel gave up; "
                                  f"{int((st == _lib.ST_TIMEOUT).sum().item())} conformers have no valid result")
        return MinimizeResult(pos_dev.cpu().numpy(), e.cpu().numpy(), st.cpu().numpy(), it.cpu().numpy(),
                              e64.cpu().numpy(), de.cpu().numpy(), gr.cpu().numpy())

    def fp64_check_device(self, pos_dev, energy_dev, mode=MODE_TG, stream=None):
        """FP64 energy, error of ``energy_dev`` against it, and FP64 RMS gradient of every
        conformer at ``pos_dev`` (device tensors, stream-ordered)."""
        torch = _torch()
        L = _lib.load()
        C = self.confs.n_conf
        e64 = torch.empty(C, dtype=torch.float64, device=self.batch.device)
        de = torch.empty(C, dtype=torch.float64, device=self.batch.device)
        gr = torch.empty(C, dtype=torch.float64, device=self.batch.device)
        md = (ctypes.c_double * 4)(*[float(v) for v in mode])
        bd, cd = self.batch.desc(), self.confs.desc()
        rc = L.mmffb_fp64_check(ctypes.byref(bd), ctypes.byref(cd), md, pos_dev.data_ptr(), energy_dev.data_ptr(),
                                e64.data_ptr(), de.data_ptr(), gr.data_ptr(), _stream_ptr(torch, stream))
        _lib.check(rc, "mmffb_fp64_check")
        return e64, de, gr

    def plain_minimize(self, positions: np.ndarray, *, max_iters: int, grad_tol: float = 1e-4,
                       consts=TG_CONSTS, mode=MODE_TG) -> MinimizeResult:
        """The reference design restated (32 threads per conformer, serial gradient, global H)."""
        torch = _torch()
        L = _lib.load()
        pos_dev = torch.from_numpy(np.ascontiguousarray(positions, np.float32).reshape(-1).copy()).to(
            self.batch.device)
        out = self.plain_device(pos_dev, max_iters=max_iters, grad_tol=grad_tol, consts=consts, mode=mode)
        torch.cuda.synchronize()
        e, st, it = out
        return MinimizeResult(pos_dev.cpu().numpy(), e.cpu().numpy(), st.cpu().numpy(), it.cpu().numpy())

    def plain_device(self, pos_dev, *, max_iters: int, grad_tol: float = 1e-4, consts=TG_CONSTS,
                     mode=MODE_TG, stream=None):
        torch = _torch()
        L = _lib.load()
        C = self.confs.n_conf
        plain_confs = DeviceConformers(self.batch, self.conf_mol, self.conf_coord, None)
        bd, cd = self.batch.desc(), plain_confs.desc()
        o = opt_params(max_iters, grad_tol, 0, "fp32", consts, mode)
        nbytes = L.mmffb_plain_scratch_bytes(ctypes.byref(bd), ctypes.byref(cd))
        scratch = self._scratch_for(nbytes)
        e = torch.empty(C, dtype=torch.float64, device=self.batch.device)
        st = torch.empty(C, dtype=torch.int32, device=self.batch.device)
        it = torch.empty(C, dtype=torch.int32, device=self.batch.device)
        rc = L.mmffb_plain_minimize(ctypes.byref(bd), ctypes.byref(cd), ctypes.byref(o), pos_dev.data_ptr(),
                                    e.data_ptr(), st.data_ptr(), it.data_ptr(), scratch.data_ptr(),
                                    scratch.numel(), _stream_ptr(torch, stream))
        _lib.check(rc, "mmffb_plain_minimize")
        return e, st, it

    def energy_grad(self, positions: np.ndarray, precision: str = "mixed", mode=MODE_TG, want_grad=True):
        """Energy (float64) and gradient (float32, flat) of every conformer."""
        torch = _torch()
        L = _lib.load()
        pos_dev = torch.from_numpy(np.ascontiguousarray(positions, np.float32).reshape(-1).copy()).to(
            self.batch.device)
        C = self.confs.n_conf
        e = torch.empty(C, dtype=torch.float64, device=self.batch.device)
        g = torch.zeros_like(pos_dev) if want_grad else None
        md = (ctypes.c_double * 4)(*[float(v) for v in mode])
        bd, cd = self.batch.desc(), self.confs.desc()
        rc = L.mmffb_energy_grad(ctypes.byref(bd), ctypes.byref(cd), _lib.PREC[precision], md,
                                 pos_dev.data_ptr(), e.data_ptr(), g.data_ptr() if g is not None else None,
                                 _stream_ptr(torch))
        _lib.check(rc, "mmffb_energy_grad")
        torch.cuda.synchronize()
        return e.cpu().numpy(), (g.cpu().numpy() if g is not None else None)

    def fused_sd(self, positions: np.ndarray, *, max_iters: int, max_step: float, grad_lr: float,
                 mode=MODE_MEGA):
        """Barzilai-Borwein steepest descent of the reference's fused optimizer."""
        torch = _torch()
        L = _lib.load()
        pos_dev = torch.from_numpy(np.ascontiguousarray(positions, np.float32).reshape(-1).copy()).to(
            self.batch.device)
        C = self.confs.n_conf
        e = torch.empty(C, dtype=torch.float64, device=self.batch.device)
        o = opt_params(max_iters, 0.0, 0, "mixed", TG_CONSTS, mode)
        sd = (ctypes.c_float * 2)(float(max_step), float(grad_lr))
        bd, cd = self.batch.desc(), self.confs.desc()
        rc = L.mmffb_fused_sd(ctypes.byref(bd), ctypes.byref(cd), ctypes.byref(o), sd, pos_dev.data_ptr(),
                              e.data_ptr(), _stream_ptr(torch))
        _lib.check(rc, "mmffb_fused_sd")
        torch.cuda.synchronize()
        return pos_dev.cpu().numpy(), e.cpu().numpy()


# atom-count upper bounds of the size classes.  Dense BFGS (up to 170 atoms): each class runs
# its own instance of the default plan (H in shared memory up to 24 and up to 48 atoms; the
# register-lean global-slot H to 170).  L-BFGS: up to 170 atoms the register-capped instance
# with the history in shared memory, 171-288 the register-capped one with the history in a
# global slot (both two CTAs per SM), above that the uncapped one (one CTA per SM)
DEFAULT_BINS = (24, 48, 170, 288, 1024)


class BinnedMinimizer(Minimizer):
    """Size-binned launch: conformers grouped by atom count, one launch per bin.

    Each bin gets the kernel instance that suits its molecules (small bins:
    fewer threads per conformer, inverse Hessian in shared memory, several
    CTAs per SM; large bins: 256 threads, Hessian in an L2-resident global
    slot) and its own CUDA stream, so the bins run concurrently and fill the
    SMs each other leaves idle.  ``tuning`` maps a bin's upper bound to
    {"threads": ..., "ctas_per_sm": ...} (written by ``autotune.py``).
    """

    def __init__(self, params_list, conf_counts, device=None, bins=DEFAULT_BINS, tuning=None):
        super().__init__(params_list, conf_counts, device)
        torch = _torch()
        n_atoms = np.asarray(self.batch.n_atoms, dtype=np.int64)
        nconf = n_atoms[self.conf_mol]
        self.bins = []
        self._bin_events = []
        lo = 0
        for hi in bins:
            sel = np.nonzero((nconf > lo) & (nconf <= hi))[0]
            if len(sel):
                order = sel[np.lexsort((sel, self.conf_mol[sel], -nconf[sel]))].astype(np.int32)
                dc = DeviceConformers(self.batch, self.conf_mol, self.conf_coord, order)
                dc.n_conf = len(order)          # the bin's queue: its own order array
                dc.max_atoms = int(nconf[sel].max())
                cfg = dict((tuning or {}).get(str(hi), (tuning or {}).get(hi, {})))
                self.upload_bytes += dc.nbytes
                self.bins.append({"hi": hi, "confs": dc, "n": len(order), "cfg": cfg, "sel": sel,
                                  "stream": torch.cuda.Stream(device=self.batch.device), "scratch": None,
                                  "cost": float(np.sum((3.0 * nconf[sel]) ** 2))})
            lo = hi
        # largest molecules first: their conformers take longest, so their class gets the SMs
        # first (longest-processing-time order across classes).  Launch order alone does not
        # ensure it -- the launches of the classes are queued on their streams within
        # microseconds -- so each class's stream also gets a priority, the largest molecules'
        # the highest: the block scheduler then places that class's CTAs before any other's.
        self.bins.sort(key=lambda b: -b["hi"])
        for rank, b in enumerate(self.bins):
            b["stream"] = torch.cuda.Stream(device=self.batch.device, priority=-(len(self.bins) - 1 - rank))

    def minimize_device(self, pos_dev, *, max_iters: int, grad_tol: float = 1e-4, history_m: int = 0,
                        precision: str = "mixed", consts=TG_CONSTS, mode=MODE_TG, threads: int = 0,
                        ctas_per_sm: int = 0, exit_test: int = _lib.EXIT_TG, check_every: int = 0,
                        atom_grad_scale: float = 1.0, max_restarts: int = 0, polish64=None,
                        hpass_lean: bool = True, stream=None, out=None, evals=None, err=None,
                        wait_spins: int = 0, give_up_waits: bool = False, time_bins=False):
        """As ``Minimizer.minimize_device``, one launch per size class.  With
        ``time_bins`` each launch is bracketed by timing events on its own stream;
        ``bin_times_ms()`` reads them after a synchronize."""
        torch = _torch()
        L = _lib.load()
        C = self.confs.n_conf
        if out is None:
            e = torch.empty(C, dtype=torch.float64, device=self.batch.device)
            st = torch.empty(C, dtype=torch.int32, device=self.batch.device)
            it = torch.empty(C, dtype=torch.int32, device=self.batch.device)
        else:
            e, st, it = out
        self._bin_events = []
        main = stream if stream is not None else torch.cuda.current_stream()
        fork = torch.cuda.Event()
        fork.record(main)
        bd = self.batch.desc()
        for b in self.bins:
            cfg = b["cfg"]
            o = opt_params(max_iters, grad_tol, history_m, precision, consts, mode,
                           threads or cfg.get("threads", 0), ctas_per_sm or cfg.get("ctas_per_sm", 0),
                           exit_test, check_every, atom_grad_scale, max_restarts, polish64,
                           bool(cfg.get("lean", hpass_lean)), wait_spins, 0, give_up_waits)
            cd = b["confs"].desc()
            nbytes = L.mmffb_minimize_scratch_bytes(ctypes.byref(bd), ctypes.byref(cd), ctypes.byref(o))
            if b["scratch"] is None or b["scratch"].numel() < nbytes:
                b["scratch"] = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.batch.device)
            s = b["stream"]
            s.wait_event(fork)
            if time_bins:
                t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                t0.record(s)
            rc = L.mmffb_minimize(ctypes.byref(bd), ctypes.byref(cd), ctypes.byref(o), pos_dev.data_ptr(),
                                  e.data_ptr(), st.data_ptr(), it.data_ptr(),
                                  evals.data_ptr() if evals is not None else None, b["scratch"].data_ptr(),
                                  b["scratch"].numel(), ctypes.c_void_p(s.cuda_stream))
            _lib.check(rc, "mmffb_minimize")
            if time_bins:
                t1.record(s)
                self._bin_events.append((b, t0, t1))
        for b in self.bins:
            ev = torch.cuda.Event()
            ev.record(b["stream"])
            main.wait_event(ev)
        if err is not None:
            # each size class's launch keeps its error word at byte 4 of its own scratch
            # (one shared word would be zeroed by a later class's start)
            with torch.cuda.stream(main):
                err.zero_()
                for b in self.bins:
                    err.copy_(torch.maximum(err, b["scratch"][4:8].view(torch.int32)))
        return e, st, it

    def bin_times_ms(self):
        """[(bin upper bound, conformer indices, kernel ms)] of the last ``time_bins`` call."""
        return [(b["hi"], b["sel"], t0.elapsed_time(t1)) for b, t0, t1 in self._bin_events]


def mmff_minimize_nk(
    mmff_params_list,
    conf_counts: List[int],
    positions_3d: np.ndarray,
    *,
    max_iters: int = 500,
    grad_tol: float = 1e-4,
    use_lbfgs: bool = False,
    return_result: bool = False,
):
    """Minimise N molecules x k conformers on the GPU (persistent launches per size class,
    pipelined behind the packing: ``minimize_pipelined``).

    Same signature and return values as the reference
    (mlxmolkit/mmff_minimize.py:231-346): ``positions_3d`` is the flat
    float32 coordinate array of all conformers, molecule-major; returns
    (positions float32 flat, energies float32 (C,), converged bool (C,)).
    ``use_lbfgs`` selects L-BFGS with 8 history pairs instead of dense BFGS.
    Like the reference, every call packs the molecules' tables (here on host
    threads, natively) and uploads them.  With ``return_result`` a fourth item,
    the ``MinimizeResult``, carries each conformer's status, iterations and FP64
    check (FP64 energy at the returned coordinates, the returned energy's error
    against it, FP64 RMS gradient) and the host time of each step.
    """
    r = minimize_pipelined(mmff_params_list, conf_counts, positions_3d, max_iters=max_iters,
                           grad_tol=grad_tol, history_m=LBFGS_M if use_lbfgs else 0)
    if not return_result:
        return r.positions, r.energies.astype(np.float32), r.converged
    return r.positions, r.energies.astype(np.float32), r.converged, r


_CHUNK_STREAMS: dict = {}


def _chunk_stream(device, r: int):
    """The stream of launch position r on ``device``: the same streams on every call, so the
    caching allocator reuses each position's scratch blocks (it keeps freed blocks per stream);
    priority highest for r = 0 and one level lower per position, down to the lowest."""
    torch = _torch()
    key = (str(device), r)
    s = _CHUNK_STREAMS.get(key)
    if s is None:
        lowest, highest = torch.cuda.Stream.priority_range()
        s = torch.cuda.Stream(device=device, priority=min(lowest, highest + r))
        _CHUNK_STREAMS[key] = s
    return s


def _ranges(starts, lens) -> np.ndarray:
    """The concatenated index ranges [starts[i], starts[i] + lens[i])."""
    starts = np.asarray(starts, dtype=np.int64)
    lens = np.asarray(lens, dtype=np.int64)
    if lens.size == 0:
        return np.zeros(0, dtype=np.int64)
    first = np.concatenate([[0], np.cumsum(lens)[:-1]])
    return np.repeat(starts - first, lens) + np.arange(int(lens.sum()), dtype=np.int64)


def launch_chunks(n_atoms, conf_counts, bins=DEFAULT_BINS, head_frac: float = 0.1, min_split: int = 64):
    """Molecule index groups of a pipelined call, in launch order.

    Molecules with conformers are grouped by size class (``bins``, as ``BinnedMinimizer``;
    atom counts above the last bound form a class of their own), largest class first and
    largest molecules first within a class.  The first class is split after its largest
    ``head_frac`` of molecules (when it has at least ``min_split``), so the first launch
    waits only for their packing.
    """
    n = np.asarray(n_atoms, dtype=np.int64)
    k = np.asarray(conf_counts, dtype=np.int64)
    live = np.nonzero(k > 0)[0]
    cls = np.searchsorted(np.asarray(bins, dtype=np.int64), n[live], side="left")
    chunks = []
    for c in sorted(set(cls.tolist()), reverse=True):
        mols = live[cls == c]
        mols = mols[np.lexsort((mols, -n[mols]))]
        if not chunks and len(mols) >= min_split:
            h = max(1, int(math.ceil(head_frac * len(mols))))
            chunks += [mols[:h], mols[h:]]
        else:
            chunks.append(mols)
    return chunks


def minimize_pipelined(params_list, conf_counts, positions, *, max_iters: int, grad_tol: float = 1e-4,
                       history_m: int = 0, device=None) -> MinimizeResult:
    """The drop-in call's body: pack, upload and launch chunk by chunk (``launch_chunks``).

    Chunk r is packed (native, host threads), uploaded and launched on its own stream while
    the GPU runs chunks 0..r-1; streams get priorities in launch order, so a later chunk's
    CTAs take SMs as an earlier chunk's work queue drains.  Each chunk's FP64 check and result
    copies follow its launch on the same stream, and the call returns once every chunk's
    results are on the host.

    Every chunk is planned at its size class's atom bound, and the planner picks the kernel
    instance from the atom bound alone, so a conformer's result is the same as in one
    ``BinnedMinimizer`` launch per class.

    ``timings`` holds host seconds: ``setup_s`` until the first launch, ``pack_s`` over all
    chunks (mostly overlapped with the GPU), ``minimize_s`` from the first launch to the last
    result, ``total_s``.
    """
    torch = _torch()
    t0 = time.perf_counter()
    params_list = list(params_list)
    k = np.asarray([int(c) for c in conf_counts], dtype=np.int64)
    n = np.asarray([int(p.n_atoms) for p in params_list], dtype=np.int64)
    if len(k) != len(params_list):
        raise ValueError("conf_counts needs one entry per molecule")
    pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
    sizes = 3 * n * k
    coord0 = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    conf0 = np.concatenate([[0], np.cumsum(k)]).astype(np.int64)
    if pos.size != int(coord0[-1]):
        raise ValueError(f"positions hold {pos.size} floats, the conformers need {int(coord0[-1])}")
    C = int(conf0[-1])
    chunks = launch_chunks(n, k)
    # every chunk is planned at its size class's atom bound (the largest molecule of the class),
    # as the class's one launch in BinnedMinimizer is: the same kernel instance and layout
    cls_of = [int(np.searchsorted(np.asarray(DEFAULT_BINS), n[c[0]], side="left")) for c in chunks]
    bound = {}
    for c, ci in zip(chunks, cls_of):
        bound[ci] = max(bound.get(ci, 0), int(n[c].max()))
    dev = device or torch.device("cuda", torch.cuda.current_device())
    live = []
    pack_s, upload, t_first = 0.0, 0, None
    for r, idx in enumerate(chunks):
        s = _chunk_stream(dev, r)
        with torch.cuda.stream(s):
            m = Minimizer([params_list[i] for i in idx], [int(k[i]) for i in idx], dev)
            m.confs.max_atoms = bound[cls_of[r]]
            pack_s += m.pack_s
            xh = torch.from_numpy(np.concatenate([pos[coord0[i]:coord0[i + 1]] for i in idx])).pin_memory()
            x = torch.empty(xh.numel(), dtype=torch.float32, device=dev)
            x.copy_(xh, non_blocking=True)
            err = torch.zeros(1, dtype=torch.int32, device=dev)
            e, st, it = m.minimize_device(x, max_iters=max_iters, grad_tol=grad_tol, history_m=history_m,
                                          err=err, stream=s)
            if t_first is None:
                t_first = time.perf_counter()
            e64, de, gr = m.fp64_check_device(x, e, stream=s)
            host = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in (x, e, st, it, e64, de, gr, err)]
            for h, t in zip(host, (x, e, st, it, e64, de, gr, err)):
                h.copy_(t, non_blocking=True)
            done = torch.cuda.Event()
            done.record(s)
        upload += m.upload_bytes          # tables and conformer index arrays (coordinates apart)
        live.append((idx, m, done, host, (x, e, st, it, e64, de, gr, err)))
    out_pos = np.empty(pos.size, dtype=np.float32)
    outs = [np.empty(C, dtype=np.float64), np.empty(C, dtype=np.int32), np.empty(C, dtype=np.int32),
            np.empty(C, dtype=np.float64), np.empty(C, dtype=np.float64), np.empty(C, dtype=np.float64)]
    gave_up, bad = False, 0
    for idx, m, done, host, _ in live:
        done.synchronize()
        hx, he, hst, hit, he64, hde, hgr, herr = (h.numpy() for h in host)
        out_pos[_ranges(coord0[idx], sizes[idx])] = hx
        cidx = _ranges(conf0[idx], k[idx])
        for o, h in zip(outs, (he, hst, hit, he64, hde, hgr)):
            o[cidx] = h
        if int(herr[0]):
            gave_up = True
            bad += int(np.sum(hst == _lib.ST_TIMEOUT))
    if gave_up:
        raise _lib.MMFFBError("mmffb_minimize: a bounded wait inside the kernel gave up; "
                              f"{bad} conformers have no valid result")
    t2 = time.perf_counter()
    res = MinimizeResult(out_pos, *outs)
    res.timings = {"setup_s": (t_first or t2) - t0, "pack_s": pack_s, "minimize_s": t2 - (t_first or t2),
                   "total_s": t2 - t0, "upload_bytes": int(upload), "launch_chunks": len(chunks)}
    return res
