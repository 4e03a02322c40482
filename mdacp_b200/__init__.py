"""mdacp_b200: B200-native Lennard-Jones timestep behind MDACP's interfaces.

Python access to the C ABI of ``libmdacp_b200.so`` (declared in
include/mdacp_b200.h) through ctypes.  The library is built in-tree by
``__graft_entry__.build()`` (or ``make -C mdacp_b200/csrc``); importing this
package never falls back to anything else: if the library is missing or no
CUDA device is present, constructing a ``System`` raises.
"""
from __future__ import annotations

import ctypes
import pathlib

import numpy as np

__all__ = [
    "LIB_PATH",
    "MdgError",
    "Params",
    "Info",
    "Replica",
    "AdjointParams",
    "External",
    "System",
    "Ensemble",
    "load_library",
    "FP64",
    "FP32_MIXED",
    "NVE",
    "NOSE_HOOVER",
    "LANGEVIN",
]

LIB_PATH = pathlib.Path(__file__).resolve().parent / "libmdacp_b200.so"

FP64, FP32_MIXED = 0, 1
OBSERVE_CURRENT, OBSERVE_GHOST_LAG = 0, 1
NVE, NOSE_HOOVER, LANGEVIN = 0, 1, 2

STATUS_NAMES = {
    0: "MDG_OK",
    -1: "MDG_ERR_INVALID_ARGUMENT",
    -2: "MDG_ERR_CUDA",
    -3: "MDG_ERR_CAPACITY",
    -4: "MDG_ERR_TOO_FAST",
    -5: "MDG_ERR_INVALID_POSITION",
    -6: "MDG_ERR_NONFINITE",
    -7: "MDG_ERR_BOX_TOO_SMALL",
    -8: "MDG_ERR_TIMEOUT",
    -9: "MDG_ERR_STATE",
    -10: "MDG_ERR_NO_DEVICE",
    -11: "MDG_ERR_IO",
}


class MdgError(RuntimeError):
    """A non-zero mdg_status; ``status`` holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Params(ctypes.Structure):
    """``mdg_params`` (include/mdacp_b200.h)."""

    _fields_ = [
        ("capacity", ctypes.c_int),
        ("L", ctypes.c_double * 3),
        ("cutoff", ctypes.c_double),
        ("buffer_length", ctypes.c_double),
        ("time_step", ctypes.c_double),
        ("precision", ctypes.c_int),
        ("thermostat", ctypes.c_int),
        ("aimed_temperature", ctypes.c_double),
        ("heatbath_tau", ctypes.c_double),
        ("heatbath_gamma", ctypes.c_double),
        ("seed", ctypes.c_uint64),
        ("check_list_length", ctypes.c_int),
        ("max_neighbors", ctypes.c_int),
        ("device", ctypes.c_int),
        ("stream", ctypes.c_void_p),
        ("stage_atoms", ctypes.c_int),
        ("threads_per_atom", ctypes.c_int),
        ("build_block", ctypes.c_int),
        ("build_threads_per_atom", ctypes.c_int),
        ("step_mode", ctypes.c_int),
        ("stage_wait_cycles", ctypes.c_longlong),
    ]


STEPS_AUTO, STEPS_GRAPHS, STEPS_PERSISTENT = 0, 1, 2


class Info(ctypes.Structure):
    """``mdg_info`` (include/mdacp_b200.h)."""

    _fields_ = [
        ("n", ctypes.c_int),
        ("ncell", ctypes.c_int * 3),
        ("max_neighbors", ctypes.c_int),
        ("max_row", ctypes.c_int),
        ("list_entries", ctypes.c_int64),
        ("steps", ctypes.c_int64),
        ("rebuilds", ctypes.c_int64),
        ("displacement_checks", ctypes.c_int64),
        ("simulation_time", ctypes.c_double),
        ("buffer_left", ctypes.c_double),
        ("threads_per_atom", ctypes.c_int),
        ("build_block", ctypes.c_int),
        ("build_threads_per_atom", ctypes.c_int),
        ("persistent_steps", ctypes.c_int64),
    ]

    def as_dict(self):
        return {name: (list(getattr(self, name)) if name == "ncell" else getattr(self, name))
                for name, _ in self._fields_}


class AdjointParams(ctypes.Structure):
    """Mirror of mdg_adjoint_params (include/mdacp_b200.h)."""

    _fields_ = [
        ("L", ctypes.c_double * 3),
        ("cutoff", ctypes.c_double),
        ("time_step", ctypes.c_double),
        ("epsilon", ctypes.c_double),
        ("sigma", ctypes.c_double),
        ("shell_lo", ctypes.c_double),
        ("shell_hi", ctypes.c_double),
        ("shell_width", ctypes.c_double),
        ("steps", ctypes.c_int),
        ("checkpoint_every", ctypes.c_int),
        ("threads_per_atom", ctypes.c_int),
        ("device", ctypes.c_int),
    ]


class External(ctypes.Structure):
    """Mirror of mdg_external (include/mdacp_b200.h)."""

    _fields_ = [
        ("kind", ctypes.c_int),
        ("axis", ctypes.c_int),
        ("strength", ctypes.c_double),
        ("time_step", ctypes.c_double),
        ("position", ctypes.c_double),
        ("velocity", ctypes.c_double),
        ("center", ctypes.c_double * 3),
        ("radius", ctypes.c_double),
    ]


EXTERNAL_NONE, EXTERNAL_GRAVITY, EXTERNAL_PISTON, EXTERNAL_SHELL = 0, 1, 2, 3
SNAPSHOT_CDVIEW, SNAPSHOT_CONFIGURATION = 0, 1


class Replica(ctypes.Structure):
    """``mdg_replica`` (include/mdacp_b200.h)."""

    _fields_ = [("n", ctypes.c_int), ("L", ctypes.c_double * 3), ("buffer_length", ctypes.c_double)]


# name -> (restype, argtypes)
_H = ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)
_I64P = ctypes.POINTER(ctypes.c_int64)
SIGNATURES = {
    "mdg_adjoint_default_params": (None, [ctypes.POINTER(AdjointParams)]),
    "mdg_adjoint_run": (ctypes.c_int, [ctypes.POINTER(AdjointParams), _DP, _DP, ctypes.c_int, _DP, _DP, _DP, _DP]),
    "mdg_adjoint_release": (None, []),
    "mdg_default_params": (None, [ctypes.POINTER(Params)]),
    "mdg_set_external": (ctypes.c_int, [_H, ctypes.POINTER(External)]),
    "mdg_change_scale": (ctypes.c_int, [_H, ctypes.c_double]),
    "mdg_density_grid": (ctypes.c_int, [_H, ctypes.c_double, ctypes.POINTER(ctypes.c_ubyte), ctypes.c_int64, _IP]),
    "mdg_save_checkpoint": (ctypes.c_int, [_H, ctypes.c_char_p]),
    "mdg_load_checkpoint": (ctypes.c_int, [_H, ctypes.c_char_p]),
    "mdg_snapshot_async": (ctypes.c_int, [_H, ctypes.c_char_p, ctypes.c_int]),
    "mdg_snapshot_wait": (ctypes.c_int, [_H]),
    "mdg_external_state": (ctypes.c_int, [_H, _DP, _DP]),
    "mdg_create": (ctypes.c_int, [ctypes.POINTER(Params), ctypes.POINTER(_H)]),
    "mdg_destroy": (ctypes.c_int, [_H]),
    "mdg_set_state": (ctypes.c_int, [_H, _DP, _DP, _IP, ctypes.c_int]),
    "mdg_get_state": (ctypes.c_int, [_H, _DP, _DP, _IP, ctypes.c_int]),
    "mdg_get_ids": (ctypes.c_int, [_H, _IP, ctypes.c_int]),
    "mdg_particle_number": (ctypes.c_int, [_H, _IP]),
    "mdg_make_pairlist": (ctypes.c_int, [_H]),
    "mdg_check_expired": (ctypes.c_int, [_H, _IP]),
    "mdg_update_position_half": (ctypes.c_int, [_H]),
    "mdg_calculate_force": (ctypes.c_int, [_H]),
    "mdg_heatbath_zeta": (ctypes.c_int, [_H, ctypes.c_double]),
    "mdg_heatbath_momenta": (ctypes.c_int, [_H]),
    "mdg_langevin": (ctypes.c_int, [_H]),
    "mdg_get_zeta": (ctypes.c_int, [_H, _DP]),
    "mdg_set_zeta": (ctypes.c_int, [_H, ctypes.c_double]),
    "mdg_set_control": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    "mdg_get_list": (ctypes.c_int, [_H, _IP, _IP, ctypes.c_int64, _I64P]),
    "mdg_calculate": (ctypes.c_int, [_H, ctypes.c_int]),
    "mdg_forces": (ctypes.c_int, [_H, _DP]),
    "mdg_observe": (ctypes.c_int, [_H, _DP, _DP, _DP]),
    "mdg_set_observer_mode": (ctypes.c_int, [_H, ctypes.c_int]),
    "mdg_pair_counts": (ctypes.c_int, [_H, _I64P, _I64P]),
    "mdg_get_pairs": (ctypes.c_int, [_H, _IP, _IP, ctypes.c_int64, _I64P]),
    "mdg_get_info": (ctypes.c_int, [_H, ctypes.POINTER(Info)]),
    "mdg_stream": (ctypes.c_void_p, [_H]),
    "mdg_set_graph_mode": (ctypes.c_int, [_H, ctypes.c_int]),
    "mdg_set_kernel_timing": (ctypes.c_int, [_H, ctypes.c_int]),
    "mdg_kernel_time": (ctypes.c_int, [_H, _DP, _I64P, _I64P]),
    "mdg_observe_static": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_void_p, _DP, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]),
    "mdg_ensemble_create": (ctypes.c_int, [ctypes.POINTER(Params), ctypes.c_int, ctypes.c_void_p,
                                           ctypes.POINTER(_H)]),
    "mdg_ensemble_destroy": (ctypes.c_int, [_H]),
    "mdg_ensemble_set_state": (ctypes.c_int, [_H, _DP, _DP]),
    "mdg_ensemble_get_state": (ctypes.c_int, [_H, _DP, _DP, _IP]),
    "mdg_ensemble_calculate": (ctypes.c_int, [_H, ctypes.c_int]),
    "mdg_ensemble_observe": (ctypes.c_int, [_H, _DP, _DP, _DP]),
    "mdg_ensemble_rebuilds": (ctypes.c_int, [_H, _I64P, _I64P]),
    "mdg_ensemble_set_graph_mode": (ctypes.c_int, [_H, ctypes.c_int]),
    "mdg_ensemble_stream": (ctypes.c_void_p, [_H]),
    "mdg_slabs_create": (ctypes.c_int, [ctypes.POINTER(Params), ctypes.c_int, _IP, ctypes.POINTER(_H)]),
    "mdg_slabs_destroy": (ctypes.c_int, [_H]),
    "mdg_slabs_set_state": (ctypes.c_int, [_H, _DP, _DP, _IP, ctypes.c_int]),
    "mdg_slabs_get_state": (ctypes.c_int, [_H, _DP, _DP, ctypes.c_int]),
    "mdg_slabs_calculate": (ctypes.c_int, [_H, ctypes.c_int]),
    "mdg_slabs_observe": (ctypes.c_int, [_H, _DP, _DP, _DP]),
    "mdg_slabs_forces": (ctypes.c_int, [_H, _DP, ctypes.c_int]),
    "mdg_slabs_info": (ctypes.c_int, [_H, _I64P, _I64P, _IP, _IP]),
    "mdg_slabs_last_error": (ctypes.c_char_p, [_H]),
    "mdg_set_velocities": (ctypes.c_int, [_H, _DP, ctypes.c_int]),
    "mdg_partition_replicas": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, _IP,
                                              _DP]),
    "mdg_ensemble_set_kernel_timing": (ctypes.c_int, [_H, ctypes.c_int]),
    "mdg_ensemble_kernel_time": (ctypes.c_int, [_H, _DP, _I64P, _I64P]),
    "mdg_ensemble_list_stats": (ctypes.c_int, [_H, _I64P, _I64P]),
    "mdg_last_error": (ctypes.c_char_p, [_H]),
    "mdg_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "mdg_version": (ctypes.c_char_p, []),
}

_lib = None


def load_library(path: pathlib.Path | None = None) -> ctypes.CDLL:
    """Loads ``libmdacp_b200.so`` and declares every C-ABI signature; raises
    if the library has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = pathlib.Path(path or LIB_PATH)
    if not p.exists():
        raise FileNotFoundError(f"{p} is not built; run __graft_entry__.build() or make -C mdacp_b200/csrc")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _d(a):
    return a.ctypes.data_as(_DP)


def _i(a):
    return a.ctypes.data_as(_IP)


def _pad4(x: np.ndarray) -> np.ndarray:
    out = np.zeros((x.shape[0], 4), dtype=np.float64)
    out[:, :3] = x[:, :3]
    return out


class System:
    """One handle: a periodic single-domain LJ system resident on a GPU."""

    def __init__(self, L, cutoff=2.5, time_step=0.005, capacity=None, precision=FP64,
                 thermostat=NVE, aimed_temperature=1.0, heatbath_tau=0.1, heatbath_gamma=0.1,
                 seed=0, buffer_length=0.3, check_list_length=500, max_neighbors=0, device=0,
                 stream=None, n_hint=None, stage_atoms=0, threads_per_atom=0, build_block=0,
                 build_threads_per_atom=0, step_mode=0, stage_wait_cycles=0):
        self.lib = load_library()
        p = Params()
        self.lib.mdg_default_params(ctypes.byref(p))
        p.capacity = int(capacity or n_hint or 1)
        p.L[:] = [float(x) for x in L]
        p.cutoff = float(cutoff)
        p.buffer_length = float(buffer_length)
        p.time_step = float(time_step)
        p.precision = int(precision)
        p.thermostat = int(thermostat)
        p.aimed_temperature = float(aimed_temperature)
        p.heatbath_tau = float(heatbath_tau)
        p.heatbath_gamma = float(heatbath_gamma)
        p.seed = int(seed)
        p.check_list_length = int(check_list_length)
        p.max_neighbors = int(max_neighbors)
        p.device = int(device)
        p.stream = stream
        p.stage_atoms = int(stage_atoms)
        p.threads_per_atom = int(threads_per_atom)
        p.build_block = int(build_block)
        p.build_threads_per_atom = int(build_threads_per_atom)
        p.step_mode = int(step_mode)
        p.stage_wait_cycles = int(stage_wait_cycles)
        self.params = p
        h = _H()
        st = self.lib.mdg_create(ctypes.byref(p), ctypes.byref(h))
        if st != 0:
            raise MdgError(st, self.lib.mdg_status_string(st).decode())
        self.h = h
        self.n = 0

    # -- lifecycle
    def close(self):
        if getattr(self, "h", None):
            self.lib.mdg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st):
        if st != 0:
            msg = self.lib.mdg_last_error(self.h)
            raise MdgError(st, (msg or b"").decode())

    # -- state
    def set_state(self, q, v, type_=None):
        q4 = _pad4(np.asarray(q, dtype=np.float64))
        v4 = _pad4(np.asarray(v, dtype=np.float64))
        n = q4.shape[0]
        t = None
        if type_ is not None:
            t = np.ascontiguousarray(type_, dtype=np.int32)
        self._check(self.lib.mdg_set_state(self.h, _d(q4), _d(v4), _i(t) if t is not None else None, n))
        self.n = n

    def set_state4(self, q4, v4, type_=None):
        """Uploads from caller-owned (n,4) float64 arrays without a copy."""
        n = q4.shape[0]
        t = _i(type_) if type_ is not None else None
        self._check(self.lib.mdg_set_state(self.h, _d(q4), _d(v4), t, n))
        self.n = n

    def set_velocities4(self, v4):
        """New velocities in the current slot order, (n,4) float64 (mdg_set_velocities)."""
        v4 = np.ascontiguousarray(v4, dtype=np.float64)
        self._check(self.lib.mdg_set_velocities(self.h, _d(v4), v4.shape[0]))

    def get_state4(self, q4, v4, type_=None):
        t = _i(type_) if type_ is not None else None
        self._check(self.lib.mdg_get_state(self.h, _d(q4), _d(v4), t, self.n))

    def state(self):
        """(q, v, ids) in the current slot order; ids are upload indices."""
        q4 = np.empty((self.n, 4))
        v4 = np.empty((self.n, 4))
        self._check(self.lib.mdg_get_state(self.h, _d(q4), _d(v4), None, self.n))
        return q4[:, :3].copy(), v4[:, :3].copy(), self.ids()

    def state_by_id(self):
        """(q, v) ordered by upload index."""
        q, v, ids = self.state()
        qo = np.empty_like(q)
        vo = np.empty_like(v)
        qo[ids] = q
        vo[ids] = v
        return qo, vo

    def ids(self):
        ids = np.empty(self.n, dtype=np.int32)
        self._check(self.lib.mdg_get_ids(self.h, _i(ids), self.n))
        return ids

    # -- the hot path
    def make_pairlist(self):
        self._check(self.lib.mdg_make_pairlist(self.h))

    def check_expired(self) -> bool:
        e = ctypes.c_int()
        self._check(self.lib.mdg_check_expired(self.h, ctypes.byref(e)))
        return bool(e.value)

    def update_position_half(self):
        self._check(self.lib.mdg_update_position_half(self.h))

    def calculate_force(self):
        self._check(self.lib.mdg_calculate_force(self.h))

    def calculate(self, nsteps: int = 1):
        self._check(self.lib.mdg_calculate(self.h, int(nsteps)))

    def forces(self):
        """Forces in the current slot order."""
        f4 = np.empty((self.n, 4))
        self._check(self.lib.mdg_forces(self.h, _d(f4)))
        return f4[:, :3].copy()

    def forces_by_id(self):
        f = self.forces()
        out = np.empty_like(f)
        out[self.ids()] = f
        return out

    def observe(self):
        """(sum KE, sum PE, virial) as the reference's observers return them."""
        ke, pe, vir = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mdg_observe(self.h, ctypes.byref(ke), ctypes.byref(pe), ctypes.byref(vir)))
        return ke.value, pe.value, vir.value

    def pairs(self):
        """Directed (key, partner) pairs in upload indices."""
        cnt = ctypes.c_int64()
        self._check(self.lib.mdg_get_pairs(self.h, None, None, 0, ctypes.byref(cnt)))
        k = np.empty(cnt.value, dtype=np.int32)
        p = np.empty(cnt.value, dtype=np.int32)
        self._check(self.lib.mdg_get_pairs(self.h, _i(k), _i(p), cnt.value, ctypes.byref(cnt)))
        return k, p

    def set_control(self, thermostat, aimed_temperature=1.0, heatbath_tau=0.1, heatbath_gamma=0.1):
        self._check(self.lib.mdg_set_control(self.h, int(thermostat), float(aimed_temperature),
                                             float(heatbath_tau), float(heatbath_gamma)))

    def langevin(self):
        self._check(self.lib.mdg_langevin(self.h))

    def heatbath_momenta(self):
        self._check(self.lib.mdg_heatbath_momenta(self.h))

    def heatbath_zeta(self, temperature):
        self._check(self.lib.mdg_heatbath_zeta(self.h, float(temperature)))

    def neighbor_list(self):
        """Full list in slot order: (row lengths, concatenated partner slots)."""
        cnt = ctypes.c_int64()
        self._check(self.lib.mdg_get_list(self.h, None, None, 0, ctypes.byref(cnt)))
        rows = np.empty(self.n, dtype=np.int32)
        part = np.empty(cnt.value, dtype=np.int32)
        self._check(self.lib.mdg_get_list(self.h, _i(rows), _i(part), cnt.value, ctypes.byref(cnt)))
        return rows, part

    def pair_counts(self):
        """(directed list entries within the cut-off, all list entries)."""
        a, b = ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.mdg_pair_counts(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_observer_mode(self, mode: int):
        self._check(self.lib.mdg_set_observer_mode(self.h, int(mode)))

    def zeta(self) -> float:
        z = ctypes.c_double()
        self._check(self.lib.mdg_get_zeta(self.h, ctypes.byref(z)))
        return z.value

    def info(self) -> dict:
        inf = Info()
        self._check(self.lib.mdg_get_info(self.h, ctypes.byref(inf)))
        return inf.as_dict()

    def stream(self):
        return self.lib.mdg_stream(self.h)

    def set_graph_mode(self, use_graphs: bool):
        self._check(self.lib.mdg_set_graph_mode(self.h, int(bool(use_graphs))))

    def change_scale(self, alpha):
        """MDManager::ChangeScale on the device (box and positions times alpha)."""
        self._check(self.lib.mdg_change_scale(self.h, float(alpha)))
        self.params.L[:] = [x * float(alpha) for x in self.params.L]

    def density_grid(self, grid_size):
        """Atoms per cell of BubbleHist's grid, uint8 array (nz, ny, nx)."""
        dims = (ctypes.c_int * 3)()
        g = [int(x / grid_size + 0.5) for x in self.params.L]
        out = np.zeros(g[0] * g[1] * g[2], dtype=np.uint8)
        self._check(self.lib.mdg_density_grid(self.h, float(grid_size),
                                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), out.size, dims))
        return out.reshape(dims[2], dims[1], dims[0])

    def save_checkpoint(self, path):
        """Whole state to a file (mdg_save_checkpoint)."""
        self._check(self.lib.mdg_save_checkpoint(self.h, str(path).encode()))

    def load_checkpoint(self, path):
        """Restore a checkpoint into this handle (same box and parameters);
        the trajectory continues bit for bit."""
        self._check(self.lib.mdg_load_checkpoint(self.h, str(path).encode()))
        n = ctypes.c_int()
        self._check(self.lib.mdg_particle_number(self.h, ctypes.byref(n)))
        self.n = n.value

    def snapshot_async(self, path, fmt=0):
        """Queue a text snapshot (0: .cd cdview lines, 1: .cnf configuration)."""
        self._check(self.lib.mdg_snapshot_async(self.h, str(path).encode(), int(fmt)))

    def snapshot_wait(self):
        self._check(self.lib.mdg_snapshot_wait(self.h))

    def set_external(self, kind=EXTERNAL_NONE, axis=0, strength=0.0, time_step=None, position=0.0, velocity=0.0,
                     center=(0.0, 0.0, 0.0), radius=0.0):
        """Executor applied on the device after every step (mdg_set_external)."""
        x = External()
        x.kind = int(kind)
        x.axis = int(axis)
        x.strength = float(strength)
        x.time_step = float(self.params.time_step if time_step is None else time_step)
        x.position = float(position)
        x.velocity = float(velocity)
        x.center[:] = [float(c) for c in center]
        x.radius = float(radius)
        self._check(self.lib.mdg_set_external(self.h, ctypes.byref(x)))

    def external_state(self):
        """(piston position, impulse of the last pass)."""
        pos, imp = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mdg_external_state(self.h, ctypes.byref(pos), ctypes.byref(imp)))
        return pos.value, imp.value

    def set_kernel_timing(self, on: bool):
        self._check(self.lib.mdg_set_kernel_timing(self.h, int(bool(on))))

    def kernel_time(self):
        ms = ctypes.c_double()
        fl = ctypes.c_int64()
        kl = ctypes.c_int64()
        self._check(self.lib.mdg_kernel_time(self.h, ctypes.byref(ms), ctypes.byref(fl), ctypes.byref(kl)))
        return ms.value, fl.value, kl.value


class Slabs:
    """One periodic system split into z-slabs of cell layers, one slab per
    device (mdg_slabs_*); ``devices`` lists a device per slab (default: all
    on ``device``)."""

    def __init__(self, L, nslabs, cutoff=2.5, time_step=0.005, capacity=None, precision=FP64, buffer_length=0.3,
                 check_list_length=500, device=0, devices=None, threads_per_atom=0):
        self.lib = load_library()
        p = Params()
        self.lib.mdg_default_params(ctypes.byref(p))
        p.capacity = int(capacity or 1)
        p.L[:] = [float(x) for x in L]
        p.cutoff = float(cutoff)
        p.buffer_length = float(buffer_length)
        p.time_step = float(time_step)
        p.precision = int(precision)
        p.check_list_length = int(check_list_length)
        p.device = int(device)
        p.threads_per_atom = int(threads_per_atom)
        self.nslabs = int(nslabs)
        devs = None
        if devices is not None:
            devs = np.ascontiguousarray(devices, dtype=np.int32)
        h = _H()
        st = self.lib.mdg_slabs_create(ctypes.byref(p), self.nslabs, _i(devs) if devs is not None else None,
                                       ctypes.byref(h))
        if st != 0:
            raise MdgError(st, self.lib.mdg_status_string(st).decode())
        self.h = h
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.mdg_slabs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            raise MdgError(st, (self.lib.mdg_slabs_last_error(self.h) or b"").decode())

    def set_state(self, q, v, type_=None):
        q4 = _pad4(np.asarray(q, dtype=np.float64))
        v4 = _pad4(np.asarray(v, dtype=np.float64))
        t = np.ascontiguousarray(type_, dtype=np.int32) if type_ is not None else None
        self._check(self.lib.mdg_slabs_set_state(self.h, _d(q4), _d(v4), _i(t) if t is not None else None,
                                                 q4.shape[0]))
        self.n = q4.shape[0]

    def state_by_id(self):
        q4 = np.empty((self.n, 4))
        v4 = np.empty((self.n, 4))
        self._check(self.lib.mdg_slabs_get_state(self.h, _d(q4), _d(v4), self.n))
        return q4[:, :3].copy(), v4[:, :3].copy()

    def calculate(self, nsteps=1):
        self._check(self.lib.mdg_slabs_calculate(self.h, int(nsteps)))

    def observe(self):
        ke, pe, vir = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mdg_slabs_observe(self.h, ctypes.byref(ke), ctypes.byref(pe), ctypes.byref(vir)))
        return ke.value, pe.value, vir.value

    def forces_by_id(self):
        f4 = np.empty((self.n, 4))
        self._check(self.lib.mdg_slabs_forces(self.h, _d(f4), self.n))
        return f4[:, :3].copy()

    def info(self):
        steps, rebuilds = ctypes.c_int64(), ctypes.c_int64()
        owned = np.zeros(self.nslabs, dtype=np.int32)
        ghosts = np.zeros(self.nslabs, dtype=np.int32)
        self._check(self.lib.mdg_slabs_info(self.h, ctypes.byref(steps), ctypes.byref(rebuilds), _i(owned),
                                            _i(ghosts)))
        return {"steps": steps.value, "rebuilds": rebuilds.value, "owned": owned.tolist(), "ghosts": ghosts.tolist()}


def partition_replicas(boxes, nranks, search_length=2.8):
    """Balanced assignment of independent replicas to ranks
    (mdg_partition_replicas): ``boxes`` is a list of (n_atoms, L); returns
    (owner per replica, load per rank)."""
    lib = load_library()
    nrep = len(boxes)
    reps = (Replica * max(nrep, 1))()
    for k, (n, L) in enumerate(boxes):
        reps[k].n = int(n)
        reps[k].L[:] = [float(x) for x in L]
    owner = np.zeros(max(nrep, 1), dtype=np.int32)
    load = np.zeros(nranks, dtype=np.float64)
    st = lib.mdg_partition_replicas(ctypes.cast(reps, ctypes.c_void_p), nrep, float(search_length), int(nranks),
                                    _i(owner), _d(load))
    if st != 0:
        raise MdgError(st, "mdg_partition_replicas")
    return owner[:nrep], load


class Ensemble:
    """Independent periodic replicas advanced together (mdg_ensemble_*).
    ``states`` is a list of (q, v, L) per replica; ``buffer_lengths``
    (optional, one per replica, 0 = ``buffer_length``) gives replicas their
    own BufferLength (for example from :func:`choose_margins`)."""

    def __init__(self, states, cutoff=2.5, time_step=0.005, precision=FP64, buffer_length=0.3,
                 check_list_length=500, device=0, threads_per_atom=0, buffer_lengths=None):
        self.lib = load_library()
        p = Params()
        self.lib.mdg_default_params(ctypes.byref(p))
        p.threads_per_atom = int(threads_per_atom)
        p.cutoff = float(cutoff)
        p.time_step = float(time_step)
        p.precision = int(precision)
        p.buffer_length = float(buffer_length)
        p.check_list_length = int(check_list_length)
        p.device = int(device)
        self.nrep = len(states)
        reps = (Replica * self.nrep)()
        self.sizes = []
        if buffer_lengths is not None and len(buffer_lengths) != self.nrep:
            raise ValueError("one buffer length per replica")
        for k, (q, v, L) in enumerate(states):
            reps[k].n = int(q.shape[0])
            reps[k].L[:] = [float(x) for x in L]
            reps[k].buffer_length = 0.0 if buffer_lengths is None else float(buffer_lengths[k])
            self.sizes.append(int(q.shape[0]))
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        h = _H()
        st = self.lib.mdg_ensemble_create(ctypes.byref(p), self.nrep, ctypes.cast(reps, ctypes.c_void_p),
                                          ctypes.byref(h))
        if st != 0:
            raise MdgError(st, self.lib.mdg_status_string(st).decode())
        self.h = h
        self.ntot = int(self.offsets[-1])
        q4 = np.zeros((self.ntot, 4))
        v4 = np.zeros((self.ntot, 4))
        for k, (q, v, _) in enumerate(states):
            a, b = self.offsets[k], self.offsets[k + 1]
            q4[a:b, :3] = q
            v4[a:b, :3] = v
        self._check(self.lib.mdg_ensemble_set_state(self.h, _d(q4), _d(v4)))

    def _check(self, st):
        if st != 0:
            raise MdgError(st, self.lib.mdg_status_string(st).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.mdg_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def calculate(self, nsteps):
        self._check(self.lib.mdg_ensemble_calculate(self.h, int(nsteps)))

    def set_graph_mode(self, use_graphs):
        self._check(self.lib.mdg_ensemble_set_graph_mode(self.h, int(bool(use_graphs))))

    def stream(self):
        return self.lib.mdg_ensemble_stream(self.h)

    def set_kernel_timing(self, on: bool):
        self._check(self.lib.mdg_ensemble_set_kernel_timing(self.h, int(bool(on))))

    def kernel_time(self):
        """(force ms summed, force launches, kernels launched) since timing was set."""
        ms, fl, kl = ctypes.c_double(), ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.mdg_ensemble_kernel_time(self.h, ctypes.byref(ms), ctypes.byref(fl), ctypes.byref(kl)))
        return ms.value, fl.value, kl.value

    def list_stats(self):
        """(list entries of the current lists, unordered pairs within the cut-off)."""
        le, pr = ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.mdg_ensemble_list_stats(self.h, ctypes.byref(le), ctypes.byref(pr)))
        return le.value, pr.value

    def states_by_id(self):
        """Per replica (q, v) ordered by upload index within the replica."""
        q4 = np.empty((self.ntot, 4))
        v4 = np.empty((self.ntot, 4))
        ids = np.empty(self.ntot, dtype=np.int32)
        self._check(self.lib.mdg_ensemble_get_state(self.h, _d(q4), _d(v4), _i(ids)))
        out = []
        for k in range(self.nrep):
            a, b = self.offsets[k], self.offsets[k + 1]
            q = np.empty((b - a, 3))
            v = np.empty((b - a, 3))
            q[ids[a:b]] = q4[a:b, :3]
            v[ids[a:b]] = v4[a:b, :3]
            out.append((q, v))
        return out

    def observe(self):
        ke = np.empty(self.nrep)
        pe = np.empty(self.nrep)
        vir = np.empty(self.nrep)
        self._check(self.lib.mdg_ensemble_observe(self.h, _d(ke), _d(pe), _d(vir)))
        return ke, pe, vir

    def rebuilds(self):
        r = np.empty(self.nrep, dtype=np.int64)
        s = np.empty(self.nrep, dtype=np.int64)
        self._check(self.lib.mdg_ensemble_rebuilds(self.h, r.ctypes.data_as(_I64P), s.ctypes.data_as(_I64P)))
        return r, s


from . import margins  # noqa: E402  (per-replica margin tuner; imports this package lazily)
