"""Simulation: the reference's MD driver on the device-resident engine.

Mirrors deepmd_jax/md.py:48-1091 (constructor arguments, run(), getters and
setters, report rows, error-code handling and chunked re-runs) for the
routines 'NVE' (velocity Verlet), 'NVT' (Nose-Hoover chain), 'NVT_langevin'
(BAOAB Langevin), 'NPT' (MTK
barostat, coupled axes) and, with n_bead > 1, 'NVT' / 'NPT' path-integral MD
(ring-polymer BAOAB with PILE-L; Langevin barostat), with centre-of-mass
removal, fixed atoms and the Model_Devi reporter.  All device work runs in
libdpb200.so through dpb_md_*; a chunk of steps is captured once into a CUDA
graph and replayed.
"""
from __future__ import annotations

import ctypes
from time import time

import numpy as np
import torch

from . import _lib
from .engine import DeviceModel, NeighborBuilder, sort_by_type, _ptr, _stream
from . import dump
from .md_utils import knbr_from_counts, print_run_profile
from .pimd import HBAR, normal_mode_transform, spring_energy, unwrap_across_beads
from .systems import MASS_UNIT_CONVERSION, TEMP_UNIT_CONVERSION
from .utils import load_model



class MDDesc(ctypes.Structure):
    _fields_ = [
        ("routine", ctypes.c_int), ("natoms", ctypes.c_int), ("nbeads", ctypes.c_int),
        ("type_idx", ctypes.POINTER(ctypes.c_int)), ("mass_per_type", ctypes.POINTER(ctypes.c_double)),
        ("sel", ctypes.POINTER(ctypes.c_int)), ("box", ctypes.c_double * 3), ("skin", ctypes.c_double),
        ("dt", ctypes.c_double), ("temperature", ctypes.c_double), ("chain_length", ctypes.c_int),
        ("tau_t", ctypes.c_double), ("pimd_lambda", ctypes.c_double),
        ("nm_transform", ctypes.POINTER(ctypes.c_double)), ("nm_freqs", ctypes.POINTER(ctypes.c_double)),
        ("seed", ctypes.c_uint64), ("precision", ctypes.c_int),
        ("pressure", ctypes.c_double), ("tau_p", ctypes.c_double), ("chain_length_p", ctypes.c_int),
        ("couple_groups", ctypes.c_int * 3), ("remove_com_motion", ctypes.c_int),
        ("fixed_indices", ctypes.POINTER(ctypes.c_int)), ("n_fixed", ctypes.c_int),
    ]


class MDReport(ctypes.Structure):
    _fields_ = [
        ("potential_energy", ctypes.c_double), ("kinetic_energy", ctypes.c_double),
        ("virial", ctypes.c_double * 9), ("thermostat_work", ctypes.c_double), ("status", ctypes.c_uint32),
        ("steps", ctypes.c_uint64), ("rebuilds", ctypes.c_uint64), ("rebuild_rate", ctypes.c_double),
        ("chain_length", ctypes.c_int), ("chain_dof", ctypes.c_double),
        ("chain_xi", ctypes.c_double * 8), ("chain_p", ctypes.c_double * 8), ("chain_Q", ctypes.c_double * 8),
        ("box", ctypes.c_double * 3), ("ngroups", ctypes.c_int),
        ("box_position", ctypes.c_double * 3), ("box_momentum", ctypes.c_double * 3),
        ("box_mass", ctypes.c_double * 3), ("baro_length", ctypes.c_int),
        ("baro_xi", ctypes.c_double * 8), ("baro_p", ctypes.c_double * 8), ("baro_Q", ctypes.c_double * 8),
        ("dU_deps", ctypes.c_double * 3), ("box_thermostat_work", ctypes.c_double),
    ]


def _declare(lib):
    if getattr(lib, "_md_declared", False):
        return
    vp = ctypes.c_void_p
    d64 = ctypes.POINTER(ctypes.c_double)
    lib.dpb_md_create.argtypes = [vp, ctypes.POINTER(MDDesc), ctypes.POINTER(vp)]
    lib.dpb_md_destroy.argtypes = [vp]
    lib.dpb_md_set_positions.argtypes = [vp, d64]
    lib.dpb_md_set_velocities.argtypes = [vp, d64]
    lib.dpb_md_get_state.argtypes = [vp, d64, d64, d64]
    lib.dpb_md_init.argtypes = [vp, ctypes.c_int, vp]
    lib.dpb_md_run.argtypes = [vp, ctypes.c_int, vp, vp, vp]
    lib.dpb_md_report.argtypes = [vp, ctypes.POINTER(MDReport)]
    lib.dpb_md_clear_status.argtypes = [vp, ctypes.c_uint32]
    lib.dpb_md_snapshot.argtypes = [vp, ctypes.c_int]
    lib.dpb_md_set_capacity.argtypes = [vp, ctypes.POINTER(ctypes.c_int), vp]
    lib.dpb_md_set_skin.argtypes = [vp, ctypes.c_double, vp]
    lib.dpb_md_device_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t)]
    lib.dpb_md_autotune.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_int), vp]
    lib.dpb_md_box_history.argtypes = [vp, ctypes.c_int, d64]
    lib.dpb_md_eval_model.argtypes = [vp, vp, d64, d64]
    lib.dpb_md_traj_frames.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp]
    for f in ("dpb_md_create", "dpb_md_destroy", "dpb_md_set_positions", "dpb_md_set_velocities",
              "dpb_md_get_state", "dpb_md_init", "dpb_md_run", "dpb_md_report", "dpb_md_clear_status",
              "dpb_md_snapshot", "dpb_md_set_capacity", "dpb_md_set_skin", "dpb_md_device_bytes",
              "dpb_md_autotune", "dpb_md_box_history", "dpb_md_eval_model", "dpb_md_traj_frames"):
        getattr(lib, f).restype = ctypes.c_int
    lib._md_declared = True


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def sel_from_counts(max_counts, buffer_ratio):
    """Kept columns (knbr - 1) per type under the reference's capacity rule
    (md_utils.py:394-403)."""
    return [max(k - 1, 1) for k in knbr_from_counts(max_counts, buffer_ratio)]


PRESS_UNIT_CONVERSION = 6.241509e-7  # bar -> eV / A^3 (deepmd_jax/md.py:26)


def parse_couple_axes(couple_axes):
    """Validated groups and the group of each axis (-1: fixed), as the
    reference's _parse_couple_axes (deepmd_jax/routine.py:196-229)."""
    try:
        groups = tuple(tuple(int(a) for a in g) for g in couple_axes)
    except TypeError:
        raise ValueError("couple_axes must be a tuple of tuples of ints; got %r" % (couple_axes,))
    axes = [a for g in groups for a in g]
    if any(a not in (0, 1, 2) for a in axes):
        raise ValueError("couple_axes axes must be in {0,1,2}; got %r" % (couple_axes,))
    if len(set(axes)) != len(axes):
        raise ValueError("couple_axes must be a partition (no repeats); got %r" % (couple_axes,))
    if any(len(g) == 0 for g in groups):
        raise ValueError("couple_axes groups must be non-empty; got %r" % (couple_axes,))
    if len(groups) == 0:
        raise ValueError("couple_axes must contain at least one group; use NVT instead")
    gid = [-1, -1, -1]
    for k, g in enumerate(groups):
        for a in g:
            gid[a] = k
    return groups, gid


class Simulation:
    """Two-step usage, as in the reference: ``sim = Simulation(...)`` then
    ``traj = sim.run(steps)``.  Extra keyword ``precision`` selects 'fp32'
    (default, the reference's float32) or 'mixed' (BF16 tensor-core GEMMs);
    ``autotune`` (default: on from 10,000 atom-beads) lets the library time
    its launch-shape candidates on this system once, before any graph is
    captured (``launch_shapes`` holds the choice).  Besides a model.pkl path
    or a (params, variables) pair, ``model_path`` may be a ``DeviceModel``
    already resident on the device, whose weights the engine then shares
    (the serving loop's MD continuations do this)."""

    def __init__(self, model_path, box, type_idx, mass, routine, dt, initial_position, initial_velocity=None,
                 report_interval=200, temperature=None, pressure=None, debug=False, seed=0,
                 model_deviation_paths=(), use_neighbor_list_when_possible=True, neighbor_skin=None,
                 neighbor_buffer_ratio=1.2, remove_com_motion=False, tau_t=100., tau_p=1000., chain_length_t=3,
                 chain_length_p=3, chain_steps_t=1, chain_steps_p=1, sy_steps_t=1, sy_steps_p=1,
                 fixed_indices=None, couple_axes=((0, 1, 2),), n_bead=1, type_symbols=None, pimd_lambda=1.0,
                 pimd_print_invariant=False, precision="fp32", use_cuda_graph=True, verbose=True, autotune=None):
        self.lib = _lib.load()
        _declare(self.lib)
        self.verbose = verbose
        resident = None
        if isinstance(model_path, DeviceModel):   # weights already on the device (the serving loop's)
            resident, params, variables = model_path, model_path.params, None
        elif isinstance(model_path, (tuple, list)):
            params, variables = model_path
        else:
            model, variables = load_model(model_path)
            params = model.params
        self._params = params
        # argument checks before any device work, with the reference's
        # messages (md.py:136-165,176-181,242-244,228-229,324,382-383)
        if float(pimd_lambda) < 0:
            raise ValueError("pimd_lambda must be non-negative.")
        if int(n_bead) > 1:
            if routine not in ("NVT", "NPT"):
                raise NotImplementedError(
                    "Path-integral MD (n_bead > 1) currently supports routine='NVT' or 'NPT'.")
            if fixed_indices is not None:
                raise NotImplementedError("fixed_indices is not supported with n_bead > 1.")
            if len(model_deviation_paths) > 0:
                raise NotImplementedError("model_deviation_paths is not supported with n_bead > 1.")
            if remove_com_motion:
                raise NotImplementedError("remove_com_motion is not supported with n_bead > 1.")
            if np.ndim(initial_position) not in (2, 3):
                raise ValueError("initial_position must have shape (N,3) or (P,N,3).")
        ct = params.get("chemical_types")
        if ct is not None:
            unknown = set(np.asarray(type_idx, dtype=int).tolist()) - set(ct)
            if unknown:
                raise ValueError('Atomic numbers %s in type_idx are not in model.params["chemical_types"]=%s'
                                 % (sorted(unknown), ct))
        if not (isinstance(couple_axes, tuple) and couple_axes == ((0, 1, 2),)) and "NPT" not in routine:
            raise ValueError("couple_axes is only meaningful for routine='NPT'")
        if routine not in ("NVE", "NVT", "NVT_langevin", "NPT"):
            raise NotImplementedError("routine currently limited to 'NVE', 'NVT', 'NVT_langevin', 'NPT'")
        if fixed_indices is not None and routine not in ("NVE", "NVT", "NVT_langevin"):
            raise NotImplementedError("Fixing atoms currently limited to NVE, NVT, and NVT_langevin routines.")
        if chain_steps_t != 1 or sy_steps_t != 1 or chain_steps_p != 1 or sy_steps_p != 1:
            raise NotImplementedError("Nose-Hoover chain_steps/sy_steps other than 1")
        if routine == "NPT":
            if pressure is None:
                raise ValueError("Missing argument 'pressure' (in bar) for routine 'NPT'")
            if temperature is None:
                raise ValueError("Missing argument 'temperature' for routine 'NPT'")
            self._couple_axes, self._group_ids = parse_couple_axes(couple_axes)
        self.model = resident if resident is not None else DeviceModel(params, variables)
        # models of the Model_Devi reporter (md.py:299-302,559-567): paths, or
        # (params, variables) pairs
        self._dev_models = []
        for mp in model_deviation_paths:
            if isinstance(mp, (tuple, list)):
                dp, dv = mp
            else:
                dm_, dv = load_model(mp)
                dp = dm_.params
            if int(dp["ntypes"]) != int(params["ntypes"]):
                raise ValueError("deviation model has %d types, the simulated model %d"
                                 % (int(dp["ntypes"]), int(params["ntypes"])))
            self._dev_models.append(DeviceModel(dp, dv))
        self._remove_com = bool(remove_com_motion)
        self._pimd_print_invariant = bool(pimd_print_invariant) and int(n_bead) > 1
        self._n_bead = int(n_bead)
        self._is_pimd = self._n_bead > 1
        self._pressure = pressure
        pos0 = np.asarray(initial_position, dtype=np.float64)
        if self._is_pimd:
            if pos0.ndim == 2:
                pos0 = np.broadcast_to(pos0, (self._n_bead,) + pos0.shape).copy()
            elif pos0.shape[0] != self._n_bead:
                raise ValueError("initial_position leading axis %d does not match n_bead=%d"
                                 % (pos0.shape[0], self._n_bead))
            self._natoms = pos0.shape[1]
        else:
            self._natoms = pos0.shape[0]
        box = np.asarray(box, dtype=np.float64)
        if box.size == 1:
            box = box.item() * np.ones(3)
        elif box.shape == (3, 3):
            if not np.allclose(box, np.diag(np.diag(box))):
                raise NotImplementedError("non-orthorhombic boxes are not supported")
            box = np.diag(box).copy()
        self._box = box
        self._routine = routine
        self._dt = float(dt)
        self._temperature = temperature
        self.report_interval = int(report_interval)
        self.step = 0
        self.log = []
        self._debug = debug
        self.precision = precision
        self._type_idx = np.asarray(type_idx, dtype=np.int32)
        if ct is not None:
            z2i = {z: i for i, z in enumerate(ct)}
            self._type_idx = np.array([z2i[int(z)] for z in self._type_idx], dtype=np.int32)
        if type_symbols is None and ct is not None:
            type_symbols = [dump.SYMBOLS[int(z)] for z in ct]
        if type_symbols is not None and len(type_symbols) < int(self._type_idx.max()) + 1:
            raise ValueError("type_symbols has length %d but type_idx needs %d types"
                             % (len(type_symbols), int(self._type_idx.max()) + 1))
        self._type_symbols = list(type_symbols) if type_symbols is not None else None
        self._mass_per_type = np.asarray(mass, dtype=np.float64)
        self._mass = self._mass_per_type[self._type_idx]
        self._step_chunk_size = max(10, min(100, 100000 // (self._natoms * self._n_bead)))
        self._neighbor_skin = ((0.5 if routine == "NPT" else 0.3) if neighbor_skin is None else float(neighbor_skin))
        self._buffer_ratio = float(neighbor_buffer_ratio)
        self._kT = (temperature if temperature is not None else 0.0) * TEMP_UNIT_CONVERSION
        self._use_graph = use_cuda_graph
        self._graphs = {}
        self._graph_kernels = {}
        self._graph_launches_replayed = 0
        nt = int(params["ntypes"])
        self._perm, self._type_count = sort_by_type(self._type_idx, nt)
        # neighbour capacity from a measurement at the initial positions (allocate_fn)
        self._sel = self._measure_capacity(pos0)
        desc = MDDesc()
        # NVT PIMD: PILE-L (pimd.py:114-207); NPT PIMD: Langevin barostat (pimd.py:255-518)
        # NVT_langevin: BAOAB with friction 1/tau_t (routine.py:46-107, md.py:352-356)
        desc.routine = ({"NVT": 2, "NPT": 4}[routine] if self._is_pimd
                        else {"NVE": 0, "NVT": 1, "NPT": 3, "NVT_langevin": 5}[routine])
        if routine == "NPT":
            desc.pressure = float(pressure) * PRESS_UNIT_CONVERSION
            desc.tau_p = float(tau_p)
            desc.chain_length_p = int(chain_length_p)
            for a in range(3):
                desc.couple_groups[a] = int(self._group_ids[a])
        desc.natoms = self._natoms
        desc.nbeads = self._n_bead
        desc.remove_com_motion = int(self._remove_com)
        # fixed atoms (md.py:221-236): a mobile mask; the engine masks shifts,
        # forces and momenta and gives the chain 3 n_mobile degrees of freedom
        self._mobile = None
        if fixed_indices is not None:
            self._mobile = np.ones(self._natoms, dtype=bool)
            self._mobile[np.asarray(fixed_indices, dtype=np.int64)] = False
            self._fixed_arr = np.ascontiguousarray(np.flatnonzero(~self._mobile), dtype=np.int32)
            desc.fixed_indices = self._fixed_arr.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
            desc.n_fixed = len(self._fixed_arr)
        self._keep = [np.ascontiguousarray(self._type_idx, dtype=np.int32), np.ascontiguousarray(self._mass_per_type)]
        desc.type_idx = self._keep[0].ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        desc.mass_per_type = _dptr(self._keep[1])
        self._sel_arr = (ctypes.c_int * nt)(*self._sel)
        desc.sel = self._sel_arr
        for k in range(3):
            desc.box[k] = float(box[k])
        desc.skin = self._neighbor_skin
        desc.dt = self._dt
        desc.temperature = float(temperature or 0.0)
        desc.chain_length = int(chain_length_t)
        desc.tau_t = float(tau_t)
        desc.pimd_lambda = float(pimd_lambda)
        desc.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        desc.precision = {"fp32": 0, "mixed": 1}[precision]
        if self._is_pimd:
            self._nm_freqs, self._nm_trans = normal_mode_transform(self._n_bead, self._kT)
            self._keep += [np.ascontiguousarray(self._nm_trans), np.ascontiguousarray(self._nm_freqs)]
            desc.nm_transform = _dptr(self._keep[-2])
            desc.nm_freqs = _dptr(self._keep[-1])
        self._desc = desc
        h = ctypes.c_void_p()
        _lib.check(self.lib.dpb_md_create(self.model.handle, ctypes.byref(desc), ctypes.byref(h)), "dpb_md_create")
        self._h = h
        self._set_pos(pos0)
        if initial_velocity is not None:
            vel = np.asarray(initial_velocity, dtype=np.float64)
        else:
            vel = self._initial_velocity(seed)
        self._set_vel(vel)
        _lib.check(self.lib.dpb_md_init(self._h, 1, _stream()), "dpb_md_init")
        # launch shapes from the library's autotuner (default: systems of 10,000
        # atom-beads or more, where its few timed launches are negligible)
        self.launch_shapes = None
        if autotune if autotune is not None else self._natoms * self._n_bead >= 10000:
            nlw, dtw, fst = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            _lib.check(self.lib.dpb_md_autotune(self._h, ctypes.byref(nlw), ctypes.byref(dtw), ctypes.byref(fst),
                                                _stream()), "dpb_md_autotune")
            self.launch_shapes = {"nlist_warps_per_block": nlw.value, "dT_atoms_per_block": dtw.value,
                                  "fit_ring_stages": fst.value}
        self._is_initial_state = True
        self._error_code = 0
        if verbose:
            label = ("%s PIMD run" % routine) if self._is_pimd else ("%s run" % routine)
            print("# Initialized %s with %d atoms" % (label, self._natoms))

    # ------------------------------------------------------------------ helpers
    def _measure_capacity(self, pos0):
        frames = pos0.reshape(self._n_bead, self._natoms, 3)
        pm = torch.tensor(self._perm.astype(np.int32), device="cuda")
        big = [256] * len(self._type_count)
        nb = NeighborBuilder(self._natoms, self._n_bead, self._type_count, big, self._box,
                             float(self._params["rcut"]) + self._neighbor_skin)
        p = torch.tensor(np.ascontiguousarray(frames), dtype=torch.float32, device="cuda")
        counts = torch.empty((self._n_bead, self._natoms, len(big)), dtype=torch.int32, device="cuda")
        nb.build(p, perm=pm, counts=counts)
        mx = counts.reshape(-1, len(big)).max(0).values.cpu().numpy()
        return sel_from_counts(mx, self._buffer_ratio)

    def _initial_velocity(self, seed):
        """Maxwell-Boltzmann momenta sqrt(m kT) N(0,1) with the mean momentum
        removed (jax_md initialize_momenta); PIMD beads at P kT
        (pimd.py:72-79).  numpy's generator replaces jax.random."""
        if self._kT == 0:
            return np.zeros((self._n_bead, self._natoms, 3) if self._is_pimd else (self._natoms, 3))
        rng = np.random.default_rng(seed)
        m = (self._mass * MASS_UNIT_CONVERSION)[:, None]
        if self._is_pimd:
            p = np.sqrt(m * self._kT * self._n_bead) * rng.normal(size=(self._n_bead, self._natoms, 3))
        else:
            p = np.sqrt(m * self._kT) * rng.normal(size=(self._natoms, 3))
            p = p - p.mean(0, keepdims=True)
        return p / m

    def _set_pos(self, pos):
        a = np.ascontiguousarray(np.asarray(pos, dtype=np.float64).reshape(-1))
        _lib.check(self.lib.dpb_md_set_positions(self._h, _dptr(a)), "dpb_md_set_positions")

    def _set_vel(self, vel):
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(vel, dtype=np.float64),
                                                 (self._n_bead, self._natoms, 3)).reshape(-1))
        _lib.check(self.lib.dpb_md_set_velocities(self._h, _dptr(a)), "dpb_md_set_velocities")

    def _report_struct(self):
        r = MDReport()
        _lib.check(self.lib.dpb_md_report(self._h, ctypes.byref(r)), "dpb_md_report")
        return r

    def _frame_shape(self):
        return (self._n_bead, self._natoms, 3) if self._is_pimd else (self._natoms, 3)

    def _run_chunk(self, n, traj_p, traj_v):
        stream = torch.cuda.current_stream()
        if not self._use_graph:
            _lib.check(self.lib.dpb_md_run(self._h, n, _ptr(traj_p), _ptr(traj_v), _stream()), "dpb_md_run")
            return
        key = (n, traj_p.data_ptr() if traj_p is not None else 0)
        g = self._graphs.get(key)
        if g is None:
            g = torch.cuda.CUDAGraph()
            side = torch.cuda.Stream()
            side.wait_stream(stream)
            k0 = self.lib.dpb_kernel_launch_count()
            with torch.cuda.stream(side):
                with torch.cuda.graph(g, stream=side, capture_error_mode="relaxed"):
                    rc = self.lib.dpb_md_run(self._h, n, _ptr(traj_p), _ptr(traj_v),
                                             ctypes.c_void_p(side.cuda_stream))
            stream.wait_stream(side)
            _lib.check(rc, "dpb_md_run (capture)")
            self._graphs[key] = g
            self._graph_kernels[key] = int(self.lib.dpb_kernel_launch_count() - k0)
        g.replay()
        self._graph_launches_replayed += self._graph_kernels.get(key, 0)

    # ------------------------------------------------------------------ reports
    def _report_row(self, tic):
        r = self._report_struct()
        KE = r.kinetic_energy / self._n_bead ** 2 if self._is_pimd else r.kinetic_energy
        PE = r.potential_energy / self._n_bead
        T = 2 * r.kinetic_energy / (3 * self._natoms * self._n_bead) / TEMP_UNIT_CONVERSION / self._n_bead
        if self._mobile is not None:  # md.py:478: temperature over the mobile degrees of freedom
            T *= self._natoms / int(self._mobile.sum())
        row = [self.step, T, KE, PE]
        headers = ["Step", "Temperature", "KE", "PE"]
        if self._routine == "NVE":
            row.append(KE + PE)
            headers.append("Invariant")
        elif self._routine == "NVT_langevin":  # md.py:506-511: KE + PE - thermostat work
            row.append(KE + PE - r.thermostat_work)
            headers.append("Invariant")
        elif self._routine == "NVT" and not self._is_pimd:
            kT = self._kT
            E = PE + KE + r.chain_p[0] ** 2 / (2 * r.chain_Q[0]) + r.chain_dof * kT * r.chain_xi[0]
            for k in range(1, r.chain_length):
                E += r.chain_p[k] ** 2 / (2 * r.chain_Q[k]) + kT * r.chain_xi[k]
            row.append(E)
            headers.append("Invariant")
        elif self._routine == "NPT" and not self._is_pimd:
            # Pressure (md_utils.py:139-159), moving box axes and the invariant (routine.py:439-456)
            kT = self._kT
            box = np.array(r.box)
            V = float(np.prod(box))
            dU_iso = -(r.virial[0] + r.virial[4] + r.virial[8])
            row.append((self._natoms * kT - dU_iso / 3.0) / V / PRESS_UNIT_CONVERSION)
            headers.append("Pressure")
            for a in sorted(a for g in self._couple_axes for a in g):
                row.append(box[a])
                headers.append("box_" + "xyz"[a])
            E = PE + KE + r.chain_p[0] ** 2 / (2 * r.chain_Q[0]) + r.chain_dof * kT * r.chain_xi[0]
            for k in range(1, r.chain_length):
                E += r.chain_p[k] ** 2 / (2 * r.chain_Q[k]) + kT * r.chain_xi[k]
            for k in range(r.baro_length):
                E += r.baro_p[k] ** 2 / (2 * r.baro_Q[k]) + kT * r.baro_xi[k]
            E += self._pressure * PRESS_UNIT_CONVERSION * V
            E += sum(r.box_momentum[g] ** 2 / (2 * r.box_mass[g]) for g in range(r.ngroups))
            row.append(E)
            headers.append("Invariant")
        elif self._routine == "NPT":
            # PIMD: the pressure of the bead-averaged potential (md_utils.py:139-159,
            # md.py:524) and the moving box axes (md.py:525-531)
            box = np.array(r.box)
            V = float(np.prod(box))
            dU_iso = -(r.virial[0] + r.virial[4] + r.virial[8]) / self._n_bead
            row.append((self._natoms * self._kT - dU_iso / 3.0) / V / PRESS_UNIT_CONVERSION)
            headers.append("Pressure")
            for a in sorted(a for g in self._couple_axes for a in g):
                row.append(box[a])
                headers.append("box_" + "xyz"[a])
            if self._pimd_print_invariant:
                row.append(self._pimd_invariant(r))
                headers.append("Invariant")
        elif self._routine == "NVT" and self._pimd_print_invariant:
            row.append(self._pimd_invariant(r))
            headers.append("Invariant")
        if self._dev_models:  # md.py:559-567: max over atoms and axes of the std over models
            row.append(self.model_deviation())
            headers.append("Model_Devi")
        self.log_headers = headers + ["Time"]
        row.append(time() - tic)
        headers.append("Time")
        if self.verbose:
            if not self.log:
                print(" ".join("%-12s" % h for h in headers))
            print("%-8d " % row[0] + " ".join("%-12.3f" % v for v in row[1:]))
        self.log.append(row)
        return r

    def _pimd_invariant(self, r):
        """Ring-polymer invariant (deepmd_jax/md.py:512-557): (KE + sum of
        the bead energies + spring energy - thermostat work) / P, plus under
        NPT the box kinetic energy, P_target V and minus the box thermostat
        work.  Spring energy 0.5 m omega_P^2 sum (R_b - R_{b-1})^2 over beads
        unwrapped onto bead 0's image (pimd.py:82-89,210-227), omega_P = P kT
        / hbar; float64 on the host from the engine's state."""
        P = self._n_bead
        box = np.array(r.box) if self._routine == "NPT" else np.asarray(self._box, dtype=np.float64)
        m = (self._mass * MASS_UNIT_CONVERSION)[:, None]
        spring = spring_energy(self.getPosition(), m, box, P * self._kT / HBAR)
        inv = (r.kinetic_energy + r.potential_energy + spring - r.thermostat_work) / P
        if self._routine == "NPT":
            inv += sum(0.5 * r.box_momentum[g] ** 2 / r.box_mass[g] for g in range(r.ngroups))
            inv += self._pressure * PRESS_UNIT_CONVERSION * float(np.prod(box)) - r.box_thermostat_work
        return inv

    # ------------------------------------------------------------------ public API
    def run(self, steps, dump_interval=None, dump_prefix=None, dump_content="positions", dump_mode="overwrite",
            trajectory=True):
        """Run ``steps`` steps; returns the trajectory dict of every step
        (deepmd_jax/md.py:874-964).  ``trajectory=False`` keeps every frame on
        the device (no per-step copy to the host) and returns None; the state
        stays readable through the getters."""
        dumps, interval = dump.prepare(self._type_idx, self._type_symbols, self._n_bead, self.report_interval,
                                       dump_interval, dump_prefix, dump_content, dump_mode)
        if dumps:
            trajectory = False                  # frames stream to the files instead (md.py:907-938)
        steps = int(steps)
        first = self._is_initial_state
        L = steps + int(first)
        fs = self._frame_shape()
        traj = None
        if trajectory:
            try:
                traj = {"position": np.zeros((L,) + fs), "velocity": np.zeros((L,) + fs),
                        "box": np.tile(self._box, (L, 1))}
            except MemoryError:  # md.py:849-850
                raise MemoryError("Trajectory too large to fit in CPU RAM. Please pass dump_prefix=... to stream "
                                  "to disk, or split into multiple shorter runs.")
        if first and trajectory:
            traj["position"][0] = self.getPosition()
            traj["velocity"][0] = self.getVelocity()
        tic_run = tic = time()
        if first:
            self._report_row(tic)
        if dumps and first and self.step % interval == 0:
            dump.write_frame(dumps, self.getPosition(), self.getVelocity(),
                             self.getCentroidPosition() if self._is_pimd else None, self.getBox(), step=self.step)
        self._is_initial_state = False
        NF3 = self._natoms * self._n_bead * 3
        cap = self._step_chunk_size
        if getattr(self, "_traj_bufs", None) is None:
            # two sets of trajectory frames of one chunk (chunk k is copied out
            # while chunk k + 1 runs), kept across runs so captured graphs stay valid
            self._traj_bufs = [(torch.empty((cap, NF3), dtype=torch.float32, device="cuda"),
                                torch.empty((cap, NF3), dtype=torch.float32, device="cuda")) for _ in range(2)]
        buf_p, buf_v = self._traj_bufs[0]
        which = 0
        pending = None  # an accepted chunk whose frames are still on the device
        done, idx = 0, int(first)
        overflow_twice = False
        stop = False
        while done < steps and not stop:
            n = min(self.report_interval - self.step % self.report_interval, self._step_chunk_size, steps - done)
            _lib.check(self.lib.dpb_md_snapshot(self._h, 0), "dpb_md_snapshot")
            if trajectory:
                buf_p, buf_v = self._traj_bufs[which]
            if trajectory or dumps:
                self._run_chunk(n, buf_p[:n], buf_v[:n])
            else:
                self._run_chunk(n, None, None)
            if pending is not None:  # the previous chunk's frames leave while this one runs
                self._copy_out(pending, traj)
                pending = None
            r = self._report_struct()
            code = int(r.status)
            # the reference's accumulated error word (md.py:906-916): bit 4 marks
            # a chunk re-run after one neighbour reallocation
            ec = code | (4 if overflow_twice else 0)
            if ec & 16:
                # NaN / Inf: this chunk is the last one (md.py:909-911); it is
                # still recorded below unless a hard overflow discards it
                print("# Warning: Nan or Inf encountered in simulation. Terminating.")
                self._error_code = ec
                stop = True
            if ec not in (0, 4, 16):
                if code & 1:
                    # box shrank past the skin: a larger skin, a list on the current box, re-run (md.py:649-654)
                    _lib.check(self.lib.dpb_md_snapshot(self._h, 1), "dpb_md_snapshot(restore)")
                    self._neighbor_skin += 0.4
                    _lib.check(self.lib.dpb_md_set_skin(self._h, self._neighbor_skin, _stream()), "dpb_md_set_skin")
                    _lib.check(self.lib.dpb_md_clear_status(self._h, ~1 & 0xFFFFFFFF), "dpb_md_clear_status")
                    self._graphs = {}
                    if self.verbose:
                        print("# Box shrank past the skin: neighbour skin now %.2f A" % self._neighbor_skin)
                elif code & 2:
                    # reallocate (grow the buffer ratio on a repeat) and re-run the chunk (md.py:657-668,913-916)
                    _lib.check(self.lib.dpb_md_snapshot(self._h, 1), "dpb_md_snapshot(restore)")
                    if overflow_twice:
                        self._buffer_ratio += 0.05
                    overflow_twice = True
                    self._resize_capacity()
                else:
                    # NaN after a reallocation (error word 20): the reference
                    # resolves, clears the word and leaves without this chunk
                    _lib.check(self.lib.dpb_md_snapshot(self._h, 1), "dpb_md_snapshot(restore)")
                    overflow_twice = False
                continue
            overflow_twice = False
            boxes = self._box_history(n)
            if dumps:
                self._write_dump_frames(dumps, interval, buf_p, buf_v, n, boxes)
            if not trajectory:
                done += n
                self.step += n
                if self.step % self.report_interval == 0 or done == steps:
                    self._report_row(tic)
                    tic = time()
                continue
            traj["box"][idx:idx + n] = boxes
            pending = (buf_p, buf_v, n, idx, self._chunk_event())
            which ^= 1
            idx += n
            done += n
            self.step += n
            if self.step % self.report_interval == 0 or done == steps:
                self._report_row(tic)
                tic = time()
        if pending is not None:
            self._copy_out(pending, traj)
        elapsed = time() - tic_run
        if self.verbose:  # md.py:953,966-967
            print_run_profile(steps, max(elapsed, 1e-9), self._natoms * self._n_bead, self._dt)
        if self._is_pimd and traj is not None:
            traj["centroid"] = np.stack([self._centroid(p, b) for p, b in zip(traj["position"], traj["box"])])
        return traj

    def _chunk_event(self):
        """An event on the main stream after the chunk just launched: the
        side-stream copy of its frames waits on it."""
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream())
        return ev

    def _copy_out(self, pending, traj):
        """Frames of one accepted chunk into the host trajectory: user order
        and velocities = momenta / (m * unit) in float64, formed on the device
        by dpb_md_traj_frames on a side stream (the next chunk keeps the main
        stream busy), then copied into traj[idx:idx + n].  Same values as
        un-permuting and dividing on the host (_unpack_frame): float32 ->
        float64 is exact and IEEE division is correctly rounded on both."""
        buf_p, buf_v, n, idx, ev = pending
        if getattr(self, "_copy_stream", None) is None:
            self._copy_stream = torch.cuda.Stream()
            shape = (self._step_chunk_size, self._natoms * self._n_bead * 3)
            self._frames64 = (torch.empty(shape, dtype=torch.float64, device="cuda"),
                              torch.empty(shape, dtype=torch.float64, device="cuda"))
        cs = self._copy_stream
        pos, vel = self._frames64
        with torch.cuda.stream(cs):
            cs.wait_event(ev)
            _lib.check(self.lib.dpb_md_traj_frames(self._h, n, _ptr(buf_p), _ptr(buf_v), _ptr(pos), _ptr(vel),
                                                   ctypes.c_void_p(cs.cuda_stream)), "dpb_md_traj_frames")
            dst_p, dst_v = traj["position"][idx:idx + n], traj["velocity"][idx:idx + n]
            torch.from_numpy(dst_p).copy_(pos[:n].view(dst_p.shape))
            torch.from_numpy(dst_v).copy_(vel[:n].view(dst_v.shape))
        cs.synchronize()

    def _unpack_frame(self, p_row, v_row):
        """User-order positions and velocities of one device frame row."""
        P, N = self._n_bead, self._natoms
        p = p_row.view(P, N, 3).cpu().numpy().astype(np.float64)
        m = v_row.view(P, N, 3).cpu().numpy().astype(np.float64)
        pos, mom = np.empty_like(p), np.empty_like(m)
        pos[:, self._perm] = p
        mom[:, self._perm] = m
        vel = mom / (self._mass * MASS_UNIT_CONVERSION)[None, :, None]
        return (pos, vel) if self._is_pimd else (pos[0], vel[0])

    def _write_dump_frames(self, dumps, interval, buf_p, buf_v, n, boxes):
        """Frames of the last chunk whose step is a multiple of the dump
        interval, copied from the device and appended to the XYZ files with
        the box of their step."""
        for i in range(n):
            step = self.step + i + 1
            if step % interval:
                continue
            pos, vel = self._unpack_frame(buf_p[i], buf_v[i])
            cen = self._centroid(pos, boxes[i]) if self._is_pimd else None
            dump.write_frame(dumps, pos, vel, cen, boxes[i], step=step)

    def _box_history(self, n):
        """(n, 3) box after each step of the last chunk (md.py:784-803): the
        barostat's boxes under NPT, else the fixed box."""
        if self._routine != "NPT":
            return np.tile(self._box, (n, 1))
        out = np.empty(n * 3)
        _lib.check(self.lib.dpb_md_box_history(self._h, n, _dptr(out)), "dpb_md_box_history")
        return out.reshape(n, 3)

    def _resize_capacity(self):
        pos = self.getPosition()
        self._sel = self._measure_capacity(pos)
        arr = (ctypes.c_int * len(self._sel))(*self._sel)
        _lib.check(self.lib.dpb_md_set_capacity(self._h, arr, _stream()), "dpb_md_set_capacity")
        _lib.check(self.lib.dpb_md_clear_status(self._h, ~2 & 0xFFFFFFFF), "dpb_md_clear_status")
        self._graphs = {}
        if self.verbose:
            print("# Neighborlist reallocated with size %s" % (self._sel,))

    def _centroid(self, R, box=None):
        return unwrap_across_beads(R, self._box if box is None else box).mean(0)

    def _state(self):
        shape = (self._n_bead * self._natoms * 3,)
        p, v, f = np.empty(shape), np.empty(shape), np.empty(shape)
        _lib.check(self.lib.dpb_md_get_state(self._h, _dptr(p), _dptr(v), _dptr(f)), "dpb_md_get_state")
        fs = self._frame_shape()
        return p.reshape(fs), v.reshape(fs), f.reshape(fs)

    def getPosition(self):
        return self._state()[0]

    def getVelocity(self):
        return self._state()[1]

    def getForce(self):
        return self._state()[2]

    def getCentroidPosition(self):
        p = self.getPosition()
        return self._centroid(p, self.getBox()) if self._is_pimd else p

    def getBox(self):
        """Current box (3,); under NPT the barostat's box."""
        if self._routine == "NPT":
            return np.array(self._report_struct().box)
        return np.array(self._box)

    def getEnergy(self):
        r = self._report_struct()
        return r.potential_energy / self._n_bead

    def getVirial(self):
        return np.array(self._report_struct().virial).reshape(3, 3)

    def setPosition(self, position, box=None):
        """Set the positions (deepmd_jax/md.py:984-1015): (N, 3), or (P, N, 3)
        / (N, 3) broadcast over beads; forces follow at once.  A new box is
        refused outside NPT as in the reference; under NPT the device-side
        barostat box is not reset from the host, so a box change raises
        NotImplementedError (after the reference's own checks)."""
        pos = np.asarray(position, dtype=np.float64)
        if self._is_pimd and pos.ndim == 2:
            pos = np.broadcast_to(pos, self._frame_shape())
        if pos.shape != self._frame_shape():
            raise ValueError("Position must have the same shape as the initial position, "
                             "or you have to create a new Simulation instance.")
        if box is not None:
            if "NPT" not in self._routine:
                raise ValueError("Box can only be changed in NPT simulations.")
            box = np.asarray(box, dtype=np.float64)
            if box.size == 1:
                box = box.item() * np.ones(3)
            cur = self.getBox()
            if box.shape != cur.shape:
                raise ValueError("Box must have the same shape as the initial box.")
            if not np.allclose(box, cur * (box[0] / cur[0]), rtol=1e-4, atol=1e-6):
                raise ValueError("Only isotropic box fluctuations are allowed in the current implementation.")
            raise NotImplementedError("setPosition(box=...) under NPT is not supported by the device engine")
        self._set_pos(pos)
        _lib.check(self.lib.dpb_md_init(self._h, 0, _stream()), "dpb_md_init")
        if int(self._report_struct().status) & 2:
            # the list overflowed its capacity at the new positions: re-measure
            # the capacity and recompute the forces on the full list, as the
            # reference's _keep_nbr_or_lattice_up_to_date / _resolve_error_code
            # do before its force call (md.py:1010-1015)
            self._resize_capacity()
            _lib.check(self.lib.dpb_md_init(self._h, 0, _stream()), "dpb_md_init")

    def setVelocity(self, velocity):
        self._set_vel(velocity)

    def setRandomVelocity(self, temperature, remove_com_motion=True, seed=None):
        """Maxwell-Boltzmann velocities at temperature (K), each bead at
        n_bead kT (deepmd_jax/md.py:1033-1047); numpy's generator stands in
        for jax.random."""
        if seed is None:
            seed = np.random.randint(1, 1000000)
        kT = temperature * TEMP_UNIT_CONVERSION
        m = (self._mass * MASS_UNIT_CONVERSION)[:, None]
        vel = np.random.default_rng(seed).normal(size=self._frame_shape()) * np.sqrt(kT * self._n_bead / m)
        self.setVelocity(vel)
        if remove_com_motion:
            self.remove_com_motion()

    def remove_com_motion(self):
        """Remove the centre-of-mass velocity (deepmd_jax/md.py:744-757; under
        PIMD over all beads and atoms)."""
        vel = self.getVelocity()
        m = (self._mass * MASS_UNIT_CONVERSION)[:, None]
        if self._is_pimd:
            vel = vel - (vel * m).sum(axis=(0, 1)) / (m.sum() * self._n_bead)
        else:  # over the mobile atoms (md.py:755-756); setVelocity masks the fixed ones
            mm = m * self._mobile[:, None] if self._mobile is not None else m
            vel = vel - (vel * mm).sum(0) / mm.sum()
        self.setVelocity(vel)

    def _deviation_forces(self):
        """Forces (n_models, N, 3) of the deviation models on the current
        positions, box and neighbour list."""
        out = []
        for dm in self._dev_models:
            e = np.zeros(1)
            f = np.zeros(self._natoms * 3)
            _lib.check(self.lib.dpb_md_eval_model(self._h, dm.handle, _dptr(e), _dptr(f)), "dpb_md_eval_model")
            out.append(f.reshape(self._natoms, 3))
        return np.stack(out)

    def model_deviation(self):
        """Model_Devi of the current state (deepmd_jax/md.py:559-567): the
        largest, over atoms and axes, standard deviation of the deviation
        models' forces."""
        if not self._dev_models:
            raise ValueError("no model_deviation_paths were given")
        return float(self._deviation_forces().std(axis=0).max())

    def getPressure(self):
        """Pressure (bar) of the current state: (N kT - dU/d(eps) / 3) / V with
        dU/d(eps) of the (bead-averaged) potential, -trace of the virial
        (md_utils.py:139-159, md.py:1082-1090)."""
        r = self._report_struct()
        V = float(np.prod(self.getBox()))
        dU = -(r.virial[0] + r.virial[4] + r.virial[8]) / self._n_bead
        return (self._natoms * self._kT - dU / 3.0) / V / PRESS_UNIT_CONVERSION

    def __del__(self):
        try:
            self._graphs = {}
            if getattr(self, "_h", None) is not None and self._h.value:
                self.lib.dpb_md_destroy(self._h)
        except Exception:
            pass
