"""Serving loop: continuous batching of evaluate() and MD-continuation
requests on one GPU.

The reference serves nothing: each ``evaluate()`` call (deepmd_jax/train.py:
703-788) compiles and runs its own shape, and an MD continuation is another
``Simulation.run`` (md.py:874-964, continuation semantics md.py:831-832).
Here a ``Server`` owns one device model and three worker threads:

* the admission worker moves waiting requests, first come first served, into
  service once the device bytes they will hold fit under the HBM budget;
* the evaluation worker takes every admitted ``evaluate`` request that is
  waiting (frames of any atom count and box) and runs them as ONE packed
  batch: a neighbour list per request (dpb_nlist_build) remapped into the
  packed index space (dpb_nlist_pack), then one dpb_eval_packed launch
  sequence over all frames; requests that arrive while a batch is on the GPU
  form the next batch, which the host packs while the current one runs;
* the MD worker steps every admitted MD-continuation request chunk by chunk
  (CUDA-graph replays of the device-resident engine; positions, velocities
  and thermostat state stay on the device) in round-robin, on its own CUDA
  stream, so MD chunks and evaluation batches overlap on the device; the
  engines share the server's resident weights (no model upload per
  request).  The continuations run with the library's default launch
  shapes: timing candidate shapes would cost more than a short continuation
  gains.

A request's bytes are released when it completes.  Latency is measured from
``submit_*`` to the result being ready on the host.
"""
from __future__ import annotations

import ctypes
import threading
import time
from collections import deque
from concurrent.futures import Future

import numpy as np
import torch

from . import _lib
from .engine import DeviceModel, PackedBatch, evaluate_packed
from .utils import load_model


def request_boxes(box, coord, type_idx):
    """(F, 3) float32 box lengths of an evaluate() request: one box (3,) or
    (3, 3) for every frame, or per-frame boxes in the shapes evaluate()
    takes (a leading frame axis; a (3, 3) array with three frames counts as
    three (3,) rows, as in evaluate()).  The packed batches are
    orthorhombic: a box with off-diagonal entries raises NotImplementedError
    (evaluate() takes general boxes)."""
    from .train import normalize_boxes
    F = coord.shape[0]
    box = np.asarray(box, dtype=np.float64)
    if box.shape == (3,):
        mats = np.broadcast_to(np.diag(box), (F, 3, 3))
    elif box.shape == (3, 3) and F != 3:
        mats = np.broadcast_to(box, (F, 3, 3))
    else:
        mats = normalize_boxes(coord, box, type_idx)
    diag = np.einsum("fii->fi", mats)
    if np.any(mats - diag[:, :, None] * np.eye(3) != 0):
        raise NotImplementedError("the serving loop packs orthorhombic boxes; evaluate() takes general boxes")
    return np.ascontiguousarray(diag, dtype=np.float32)


class HBMBudget:
    """Byte budget with first-come-first-served admission."""

    def __init__(self, total_bytes):
        self.total = int(total_bytes)
        self.used = 0
        self.peak = 0
        self.cv = threading.Condition()

    def try_reserve(self, n):
        with self.cv:
            if self.used + n > self.total:
                return False
            self.used += n
            self.peak = max(self.peak, self.used)
            return True

    def release(self, n):
        with self.cv:
            self.used -= n
            self.cv.notify_all()


class _Req:
    __slots__ = ("kind", "payload", "future", "t_submit", "t_start", "t_done", "bytes", "atoms", "frames")

    def __init__(self, kind, payload, nbytes, atoms, frames):
        self.kind = kind
        self.payload = payload
        self.future = Future()
        self.t_submit = time.perf_counter()
        self.t_start = None
        self.t_done = None
        self.bytes = nbytes
        self.atoms = atoms
        self.frames = frames


class Server:
    """Continuous-batching server of one se_a model on the current GPU.

    model: path of a model.pkl or (params, variables).  precision: 'fp32' or
    'mixed'.  hbm_budget: bytes of device memory the admitted requests may
    hold; a request larger than the whole budget is rejected at submission.
    sel: per-type neighbour capacity of the packed lists (doubled and the
    batch re-run on overflow).  max_batch_atoms: cap of one packed batch.
    """

    def __init__(self, model, precision="fp32", hbm_budget=60e9, sel=None, max_batch_atoms=1 << 21,
                 md_chunk=10):
        if isinstance(model, (tuple, list)):
            params, variables = model
        else:
            m, variables = load_model(model)
            params = m.params
        self.params, self.variables = params, variables
        self.precision = precision
        self.ntypes = int(params["ntypes"])
        self.rcut = float(params["rcut"])
        self.dm = DeviceModel(params, variables)
        self.sel = list(sel) if sel is not None else ([46, 92] + [46] * 4)[:self.ntypes]
        self.max_batch_atoms = int(max_batch_atoms)
        self.md_chunk = int(md_chunk)
        self.budget = HBMBudget(hbm_budget)
        self._pending = deque()
        self._eval_ready = deque()
        self._md_ready = deque()
        self._lock = threading.Condition()
        self._stop = False
        self._device = torch.cuda.current_device()
        self._eval_stream = torch.cuda.Stream()
        # pinned host staging of the evaluation batches, two of each (the batch
        # on the GPU keeps its own), allocated once: positions and the packed
        # index arrays of up to max_batch_atoms atom-frames
        self._pin = [torch.empty((self.max_batch_atoms + (1 << 16), 3), dtype=torch.float32, pin_memory=True)
                     for _ in range(2)]
        self._pin_idx = [torch.empty(3 * self.max_batch_atoms + (1 << 16), dtype=torch.int32, pin_memory=True)
                         for _ in range(2)]
        self._pin_k = 0
        self._md_stream = torch.cuda.Stream()
        self.completed = []
        self.batches = 0
        self.batch_sizes = []
        # per evaluation batch: requests, atom-frames and host seconds spent
        # packing, launching, waiting for the GPU and handing out results
        self.batch_log = []
        self._threads = []
        n = ctypes.c_size_t()
        _lib.check(self.dm.lib.dpb_eval_packed_workspace_bytes(self.dm.handle, 1024, 1, ctypes.byref(n)),
                   "dpb_eval_packed_workspace_bytes")
        self._ws_per_atom = n.value / 1024.0

    # ----------------------------------------------------------------- public
    def start(self):
        for fn in (self._admit_loop, self._eval_loop, self._md_loop):
            t = threading.Thread(target=fn, daemon=True)
            t.start()
            self._threads.append(t)
        return self

    def stop(self):
        with self._lock:
            self._stop = True
            self._lock.notify_all()
        for t in self._threads:
            t.join()
        self._threads = []

    def __enter__(self):
        return self.start()

    def __exit__(self, *a):
        self.stop()

    def submit_evaluate(self, coord, box, type_idx):
        """coord (F, N, 3) or (N, 3); box (3,), (3, 3), or per frame in any
        shape evaluate() takes ((F,), (F, 1), (F, 3), (F, 9), (F, 3, 3));
        orthorhombic only.  Returns a Future of {'energy' (F,), 'force'
        (F, N, 3), 'virial' (F, 3, 3)}."""
        coord = np.asarray(coord, dtype=np.float32)
        if coord.ndim == 2:
            coord = coord[None]
        if coord.ndim != 3 or coord.shape[2] != 3:
            raise ValueError("coord must have shape (F, N, 3) or (N, 3)")
        F, N = coord.shape[:2]
        type_idx = np.asarray(type_idx)
        if type_idx.shape != (N,):
            raise ValueError("type_idx must have one entry per atom")
        box = request_boxes(box, coord, type_idx)
        return self._submit(_Req("eval", (coord, box, type_idx), self.eval_bytes(N * F), N, F))

    def submit_md(self, position, box, type_idx, mass_per_type, steps, routine="NVT", dt=0.5, temperature=300.0,
                  velocity=None, tau_t=100.0, seed=0):
        """Continue MD of a box for ``steps`` steps on the device; returns a
        Future of {'position', 'velocity', 'energy', 'log'} at the end."""
        position = np.asarray(position, dtype=np.float64)
        N = position.shape[0]
        args = dict(position=position, box=np.asarray(box, np.float64), type_idx=np.asarray(type_idx),
                    mass_per_type=mass_per_type, steps=int(steps), routine=routine, dt=dt, temperature=temperature,
                    velocity=velocity, tau_t=tau_t, seed=seed)
        return self._submit(_Req("md", args, int(1.3 * self.eval_bytes(N)) + N * 64, N, int(steps)))

    def latency_summary(self):
        """p50 / p99 latency (s) per request kind over the completed requests."""
        out = {}
        with self._lock:
            done = list(self.completed)
        for kind in ("eval", "md"):
            rs = [r for r in done if r.kind == kind]
            lat = np.array([r.t_done - r.t_submit for r in rs])
            if len(lat):
                # queue: submit -> taken into a batch (or an MD slot); service: the rest
                q = np.array([(r.t_start if r.t_start is not None else r.t_done) - r.t_submit for r in rs])
                out[kind] = {"n": int(len(lat)), "p50_s": float(np.percentile(lat, 50)),
                             "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
                             "queue_p50_s": float(np.percentile(q, 50)), "queue_p99_s": float(np.percentile(q, 99)),
                             "service_p50_s": float(np.percentile(lat - q, 50)),
                             "service_p99_s": float(np.percentile(lat - q, 99))}
        return out

    def batch_summary(self):
        """Mean / max host seconds per evaluation batch in each phase (pack,
        launch, GPU wait, hand-out) and the mean batch size."""
        log = list(self.batch_log)
        if not log:
            return {}
        out = {"batches": len(log), "mean_requests": float(np.mean([b["requests"] for b in log])),
               "mean_atom_frames": float(np.mean([b["atoms"] for b in log]))}
        for k in ("pack_s", "launch_s", "wait_s", "handout_s"):
            v = np.array([b[k] for b in log])
            out[k] = {"mean": float(v.mean()), "max": float(v.max())}
        return out

    def eval_bytes(self, atoms):
        """Device bytes an evaluation of ``atoms`` atom-frames holds."""
        S = sum(self.sel)
        return int(atoms * (self._ws_per_atom + S * 4 + 64) + (1 << 20))

    # ----------------------------------------------------------------- internals
    def _submit(self, req):
        if req.bytes > self.budget.total:
            raise ValueError("request needs %d bytes, more than the whole HBM budget (%d)"
                             % (req.bytes, self.budget.total))
        with self._lock:
            if self._stop:
                raise RuntimeError("server stopped")
            self._pending.append(req)
            self._lock.notify_all()
        return req.future

    def _admit_loop(self):
        while True:
            with self._lock:
                while not self._stop and not self._pending:
                    self._lock.wait(0.05)
                if self._stop:
                    return
                while self._pending and self.budget.try_reserve(self._pending[0].bytes):
                    r = self._pending.popleft()
                    (self._eval_ready if r.kind == "eval" else self._md_ready).append(r)
                    self._lock.notify_all()
                blocked = bool(self._pending)
            if blocked:
                with self.budget.cv:
                    self.budget.cv.wait(0.01)

    def _finish(self, req, result=None, exc=None):
        req.t_done = time.perf_counter()
        self.budget.release(req.bytes)
        with self._lock:
            self.completed.append(req)
        if exc is not None:
            req.future.set_exception(exc)
        else:
            req.future.set_result(result)

    def _take_eval_batch(self, wait=True):
        """The admitted evaluate() requests waiting now, up to max_batch_atoms
        atom-frames; with ``wait`` block until there is one (None: stopped)."""
        with self._lock:
            while wait and not self._stop and not self._eval_ready:
                self._lock.wait(0.05)
            if not self._eval_ready:
                return None
            batch, atoms = [], 0
            while self._eval_ready and (not batch or atoms + self._eval_ready[0].atoms * self._eval_ready[0].frames
                                        <= self.max_batch_atoms):
                r = self._eval_ready.popleft()
                atoms += r.atoms * r.frames
                batch.append(r)
            return batch

    def _eval_loop(self):
        """One batch on the GPU while the host packs the next: launch batch k,
        pack batch k + 1, then wait for batch k and hand out its results."""
        torch.cuda.set_device(self._device)
        with torch.cuda.stream(self._eval_stream):
            inflight = None
            while True:
                reqs = self._take_eval_batch(wait=inflight is None)
                prep = None
                if reqs:
                    try:
                        prep = self._pack_eval_batch(reqs)
                    except Exception as ex:
                        self._fail(reqs, ex)
                if inflight is not None:
                    self._complete_eval_batch(inflight)
                    inflight = None
                if prep is not None:
                    try:
                        inflight = self._launch_eval_batch(prep)
                    except Exception as ex:
                        self._fail(prep["reqs"], ex)
                elif reqs is None and self._stop:
                    with self._lock:
                        if not self._eval_ready:
                            return

    def _fail(self, reqs, ex):
        for r in reqs:
            if not r.future.done():
                self._finish(r, exc=ex)

    def _pack_eval_batch(self, reqs):
        """Host side of a batch: the packed layout and the positions at their
        slots in one of two pinned staging buffers (alternating, so the batch
        on the GPU keeps its own)."""
        t0 = time.perf_counter()
        items, groups = [], []
        for r in reqs:
            r.t_start = t0
            coord, box, type_idx = r.payload
            F = coord.shape[0]
            start = 0
            for f in range(1, F + 1):            # frames of one request that share a box form one item
                if f == F or not np.array_equal(box[f], box[start]):
                    items.append((type_idx, f - start, box[start]))
                    groups.append((r, start, f))
                    start = f
        batch = PackedBatch(items, self.ntypes)
        self._pin_k ^= 1
        pin = self._pin[self._pin_k]
        if pin.shape[0] < batch.natoms:  # one request beyond max_batch_atoms
            pin = torch.empty((batch.natoms, 3), dtype=torch.float32, pin_memory=True)
            self._pin[self._pin_k] = pin
        slots = pin[:batch.natoms].numpy()
        slots[:] = 0.0
        for it, (r, a, b) in zip(batch.items, groups):
            n = it["natoms"] * it["nframes"]
            slots[it["slot0"]:it["slot0"] + n] = r.payload[0][a:b].reshape(-1, 3)
        return {"reqs": reqs, "batch": batch, "groups": groups, "pin": pin, "pin_idx": self._pin_idx[self._pin_k],
                "t_pack": (t0, time.perf_counter())}

    def _launch_eval_batch(self, prep):
        batch = prep["batch"]
        t0 = time.perf_counter()
        prep["pos"] = prep["pin"][:batch.natoms].to("cuda", non_blocking=True)
        prep["sel"] = list(self.sel)
        prep["out"] = evaluate_packed(self.dm, batch, prep["pos"], prep["sel"], self.rcut, self.precision,
                                      host_stage=prep["pin_idx"])
        prep["t_launch"] = (t0, time.perf_counter())
        return prep

    def _complete_eval_batch(self, prep):
        reqs, batch, groups = prep["reqs"], prep["batch"], prep["groups"]
        t_wait = time.perf_counter()
        try:
            out, sel = prep["out"], prep["sel"]
            while True:
                st = int(out["status"].item())
                if not st & 2:
                    break
                sel = [2 * s for s in sel]      # neighbour overflow: grow and re-run the batch
                self.sel = [max(a, b) for a, b in zip(self.sel, sel)]
                out = evaluate_packed(self.dm, batch, prep["pos"], sel, self.rcut, self.precision,
                                      host_stage=prep["pin_idx"])
            t_gpu = time.perf_counter()
            energy = out["energy"].cpu().numpy()
            force = out["force"].cpu().numpy()
            virial = out["virial"].cpu().numpy().reshape(-1, 3, 3)
        except Exception as ex:
            self._fail(reqs, ex)
            return
        self.batches += 1
        self.batch_sizes.append(batch.nreal)
        res = {id(r): {"energy": np.empty(r.frames), "force": np.empty((r.frames, r.atoms, 3), np.float32),
                       "virial": np.empty((r.frames, 3, 3)), "status": st} for r in reqs}
        for it, (r, a, b) in zip(batch.items, groups):
            d = res[id(r)]
            s0, n = it["seg0"], it["nframes"]
            d["energy"][a:b] = energy[s0:s0 + n]
            d["virial"][a:b] = virial[s0:s0 + n]
            d["force"][a:b] = force[it["slot0"]:it["slot0"] + n * it["natoms"]].reshape(n, it["natoms"], 3)
        for r in reqs:
            self._finish(r, res[id(r)])
        pk, ln = prep["t_pack"], prep["t_launch"]
        self.batch_log.append({"requests": len(reqs), "atoms": batch.nreal, "pack_s": pk[1] - pk[0],
                               "launch_s": ln[1] - ln[0], "wait_s": t_gpu - t_wait,
                               "handout_s": time.perf_counter() - t_gpu})

    def _md_loop(self):
        from .md import Simulation
        torch.cuda.set_device(self._device)
        active = []
        with torch.cuda.stream(self._md_stream):
            while True:
                with self._lock:
                    while not self._stop and not self._md_ready and not active:
                        self._lock.wait(0.05)
                    if self._stop and not active and not self._md_ready:
                        return
                    new = list(self._md_ready)
                    self._md_ready.clear()
                for r in new:
                    a = r.payload
                    try:
                        r.t_start = time.perf_counter()
                        sim = Simulation(self.dm, a["box"], a["type_idx"], a["mass_per_type"],
                                         a["routine"], a["dt"], a["position"], initial_velocity=a["velocity"],
                                         temperature=a["temperature"] if a["routine"] == "NVT" else None,
                                         tau_t=a["tau_t"], seed=a["seed"], report_interval=self.md_chunk,
                                         precision=self.precision, verbose=False, autotune=False)
                        active.append([r, sim, a["steps"]])
                    except Exception as ex:
                        self._finish(r, exc=ex)
                still = []
                for item in active:
                    r, sim, left = item
                    try:
                        n = min(self.md_chunk, left)
                        sim.run(n, trajectory=False)
                        item[2] = left - n
                        if item[2] == 0:
                            self._finish(r, {"position": sim.getPosition(), "velocity": sim.getVelocity(),
                                             "energy": sim.getEnergy(), "log": list(sim.log)})
                        else:
                            still.append(item)
                    except Exception as ex:
                        self._finish(r, exc=ex)
                active = still
