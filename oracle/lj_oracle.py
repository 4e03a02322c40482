"""Python access to the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Two oracles live here:

* ``Oracle``: ctypes binding of ``liblj_oracle.so``, the C restatement of the
  reference's single-domain timestep (lj_oracle.c; file:line map in lj_oracle.h).
* ``run_reference``: drives the reference MDACP itself, compiled from its own
  sources into ``oracle/_ref/`` by ``oracle/ref/build_ref.sh``, through the
  test-only ``OracleDump`` / ``OracleBench`` projects (oracle/ref/ref_harness.cc).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module; the product never does.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess
import tempfile

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "liblj_oracle.so"
REF_DIR = HERE / "_ref"

NVE, NOSE_HOOVER, LANGEVIN = 0, 1, 2


class Params(ctypes.Structure):
    _fields_ = [
        ("L", ctypes.c_double * 3),
        ("rc", ctypes.c_double),
        ("buffer_length", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("check_list_length", ctypes.c_int),
        ("thermostat", ctypes.c_int),
        ("aimed_temperature", ctypes.c_double),
        ("heatbath_tau", ctypes.c_double),
        ("heatbath_gamma", ctypes.c_double),
        ("seed", ctypes.c_uint64),
    ]


class External(ctypes.Structure):
    """Mirror of ljo_external: the reference projects' executors (gravity,
    piston, shell wall), applied after each step."""

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


_lib = None


def load_library() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        subprocess.check_call(["make", "-s", "-C", str(HERE)])
    lib = ctypes.CDLL(str(LIB_PATH))
    P = ctypes.POINTER
    dp, ip = P(ctypes.c_double), P(ctypes.c_int32)
    lib.ljo_create.restype = ctypes.c_void_p
    lib.ljo_create.argtypes = [P(Params), ctypes.c_int, dp, dp, ip]
    lib.ljo_destroy.argtypes = [ctypes.c_void_p]
    lib.ljo_make_pairlist.argtypes = [ctypes.c_void_p]
    lib.ljo_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
    for name in ("ljo_particle_number", "ljo_total_particle_number", "ljo_constructions"):
        getattr(lib, name).argtypes = [ctypes.c_void_p]
    lib.ljo_pair_number.argtypes = [ctypes.c_void_p]
    lib.ljo_pair_number.restype = ctypes.c_int64
    lib.ljo_zeta.argtypes = [ctypes.c_void_p]
    lib.ljo_zeta.restype = ctypes.c_double
    lib.ljo_get_state.argtypes = [ctypes.c_void_p, dp, dp, ip]
    lib.ljo_get_pairs.argtypes = [ctypes.c_void_p, ip, ip, ctypes.c_int64]
    lib.ljo_get_pairs.restype = ctypes.c_int64
    lib.ljo_forces.argtypes = [ctypes.c_void_p, dp]
    lib.ljo_observe.argtypes = [ctypes.c_void_p, dp, dp, dp]
    lib.ljo_observe_compensated.argtypes = [ctypes.c_void_p, dp, dp, dp]
    lib.ljo_philox4x32.argtypes = [P(ctypes.c_uint32), P(ctypes.c_uint32), P(ctypes.c_uint32)]
    lib.ljo_langevin_normals.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, dp]
    lib.ljo_apply_external.argtypes = [ctypes.c_void_p, P(External)]
    lib.ljo_apply_external.restype = ctypes.c_double
    _lib = lib
    return lib


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


class Oracle:
    """One single-domain system in the C restatement."""

    def __init__(self, q, v, ids, L, rc, dt, thermostat=NVE, temperature=1.0, tau=0.1,
                 gamma=0.1, seed=0, check_list_length=500, buffer_length=0.3):
        self.lib = load_library()
        q = np.ascontiguousarray(q, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        prm = Params()
        prm.L[:] = [float(x) for x in L]
        prm.rc = rc
        prm.buffer_length = buffer_length
        prm.dt = dt
        prm.check_list_length = check_list_length
        prm.thermostat = thermostat
        prm.aimed_temperature = temperature
        prm.heatbath_tau = tau
        prm.heatbath_gamma = gamma
        prm.seed = seed
        self.h = self.lib.ljo_create(ctypes.byref(prm), q.shape[0], _dptr(q), _dptr(v), _iptr(ids))

    def close(self):
        if self.h:
            self.lib.ljo_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def make_pairlist(self):
        if self.lib.ljo_make_pairlist(self.h) != 0:
            raise RuntimeError("oracle: MakePairList failed (invalid position or index)")

    def step(self, n):
        if self.lib.ljo_step(self.h, n) != 0:
            raise RuntimeError("oracle: step failed (too fast particle or invalid position)")

    def apply_external(self, ext: "External") -> float:
        """One executor pass (ljo_apply_external); returns the impulse."""
        return self.lib.ljo_apply_external(self.h, ctypes.byref(ext))

    @property
    def n(self):
        return self.lib.ljo_particle_number(self.h)

    @property
    def n_total(self):
        return self.lib.ljo_total_particle_number(self.h)

    @property
    def constructions(self):
        return self.lib.ljo_constructions(self.h)

    @property
    def zeta(self):
        return self.lib.ljo_zeta(self.h)

    def state(self):
        n = self.n
        q = np.empty((n, 3))
        v = np.empty((n, 3))
        ids = np.empty(n, dtype=np.int32)
        self.lib.ljo_get_state(self.h, _dptr(q), _dptr(v), _iptr(ids))
        return q, v, ids

    def pairs(self):
        """Directed (key id, partner id) pairs seen from real atoms."""
        cnt = self.lib.ljo_get_pairs(self.h, None, None, 0)
        a = np.empty(cnt, dtype=np.int32)
        b = np.empty(cnt, dtype=np.int32)
        self.lib.ljo_get_pairs(self.h, _iptr(a), _iptr(b), cnt)
        return a, b

    def forces(self):
        f = np.empty((self.n, 3))
        self.lib.ljo_forces(self.h, _dptr(f))
        return f

    def observe(self, compensated=False):
        """(KE, PE, virial) as the reference sums them; compensated=True adds
        the same terms with compensated summation (for sums over millions of
        pairs)."""
        ke = ctypes.c_double()
        pe = ctypes.c_double()
        vir = ctypes.c_double()
        fn = self.lib.ljo_observe_compensated if compensated else self.lib.ljo_observe
        fn(self.h, ctypes.byref(ke), ctypes.byref(pe), ctypes.byref(vir))
        return ke.value, pe.value, vir.value


def langevin_normals(seed, atom_id, step):
    lib = load_library()
    z = np.empty(3)
    lib.ljo_langevin_normals(seed, atom_id, step, _dptr(z))
    return z


def philox4x32(ctr, key):
    lib = load_library()
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    lib.ljo_philox4x32(c, k, o)
    return list(o)


# ---------------------------------------------------------------- reference
def reference_binary(rc: float, flavour: str = "plain") -> pathlib.Path:
    tag = {2.5: "25", 3.0: "30"}[round(rc, 3)]
    return REF_DIR / f"mdacp_rc{tag}_{flavour}"


def write_state_file(path, q, v, ids):
    q = np.ascontiguousarray(q, dtype="<f8")
    v = np.ascontiguousarray(v, dtype="<f8")
    ids = np.ascontiguousarray(ids, dtype="<i4")
    with open(path, "wb") as f:
        f.write(np.int64(q.shape[0]).tobytes())
        f.write(q.tobytes())
        f.write(v.tobytes())
        f.write(ids.tobytes())


def run_reference(mode, q, v, ids, L, rc, dt, flavour="plain", threads=1, extra=None,
                  workdir=None, timeout=3600):
    """Runs the reference binary on an injected state; returns (workdir, stdout)."""
    binary = reference_binary(rc, flavour)
    if not binary.exists():
        raise FileNotFoundError(f"{binary} not built (oracle/ref/build_ref.sh)")
    wd = pathlib.Path(workdir or tempfile.mkdtemp(prefix="mdacp_ref_"))
    wd.mkdir(parents=True, exist_ok=True)
    write_state_file(wd / "state.bin", q, v, ids)
    cfg = {
        "Mode": mode,
        "StateFile": str(wd / "state.bin"),
        "DumpPrefix": str(wd / "out"),
        "SystemSizeX": repr(float(L[0])),
        "SystemSizeY": repr(float(L[1])),
        "SystemSizeZ": repr(float(L[2])),
        "TimeStep": repr(float(dt)),
    }
    cfg.update(extra or {})
    (wd / "input.cfg").write_text("".join(f"{k}={val}\n" for k, val in cfg.items()))
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    out = subprocess.run([str(binary), "-i", str(wd / "input.cfg")], cwd=wd, env=env,
                         capture_output=True, text=True, timeout=timeout)
    if out.returncode != 0:
        raise RuntimeError(f"reference run failed ({out.returncode}):\n{out.stdout[-2000:]}\n{out.stderr[-2000:]}")
    return wd, out.stdout


def read_pair_dump(path):
    with open(path, "rb") as f:
        pn, tn = np.frombuffer(f.read(8), dtype="<i4")
        q = np.frombuffer(f.read(24 * tn), dtype="<f8").reshape(tn, 3).copy()
        typ = np.frombuffer(f.read(4 * pn), dtype="<i4").copy()
        np_ = np.frombuffer(f.read(4 * tn), dtype="<i4").copy()
        kp = np.frombuffer(f.read(4 * tn), dtype="<i4").copy()
        (total,) = np.frombuffer(f.read(8), dtype="<i8")
        sl = np.frombuffer(f.read(4 * total), dtype="<i4").copy()
    return dict(pn=int(pn), tn=int(tn), q=q, type=typ, np=np_, kp=kp, list=sl)


def read_state_dump(path):
    rec = np.dtype([("q", "<f8", 3), ("p", "<f8", 3), ("id", "<i4")])
    raw = np.fromfile(path, dtype=rec)
    return raw["q"].copy(), raw["p"].copy(), raw["id"].copy()


def read_observables(path):
    rows = {}
    for line in pathlib.Path(path).read_text().splitlines():
        parts = line.split()
        if parts[0] == "constructions":
            rows["constructions"] = float(parts[1])
            continue
        rows[parts[0]] = {parts[k]: float(parts[k + 1]) for k in range(1, len(parts) - 1, 2)}
    return rows


def reference_pairs_by_id(unit_dumps, L):
    """Directed (key id, partner id) pairs from the reference CSR of every unit.
    Ghost atoms carry no id; each is mapped to the real atom it images by a
    periodic nearest-neighbour match (distance must be below 1e-9 L)."""
    from scipy.spatial import cKDTree

    L = np.asarray(L, dtype=np.float64)
    real_q = np.concatenate([d["q"][: d["pn"]] for d in unit_dumps])
    real_id = np.concatenate([d["type"] for d in unit_dumps])
    wrapped = np.mod(real_q, L)
    tree = cKDTree(np.minimum(wrapped, np.nextafter(L, 0)), boxsize=L)
    keys, partners = [], []
    for d in unit_dumps:
        pn, tn = d["pn"], d["tn"]
        ids_all = np.empty(tn, dtype=np.int64)
        ids_all[:pn] = d["type"]
        if tn > pn:
            g = np.minimum(np.mod(d["q"][pn:], L), np.nextafter(L, 0))
            dist, idx = tree.query(g)
            if not np.all(dist < 1e-9 * L.max()):
                raise AssertionError("ghost without a matching real atom")
            ids_all[pn:] = real_id[idx]
        rows = np.repeat(np.arange(tn), d["np"])
        cols = d["list"]
        a = rows
        b = cols
        both_real = (a < pn) & (b < pn)
        # real-real pairs are seen from both atoms; real-ghost from the real one
        k1 = ids_all[a]
        p1 = ids_all[b]
        keys += [k1, p1[both_real]]
        partners += [p1, k1[both_real]]
        # a pair whose key is a ghost cannot occur (keys are min index, ghost-ghost skipped)
        assert np.all(a < pn)
    return np.concatenate(keys).astype(np.int32), np.concatenate(partners).astype(np.int32)
