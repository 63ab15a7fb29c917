"""ctypes front-end for the two CPU parity oracles (TEST INFRASTRUCTURE ONLY).

* ``kind="port"`` loads ``oracle/libtdlb_oracle.so``: the C restatement of the
  reference's time step (``oracle/tdlb_oracle.c``), OpenMP-parallel.
* ``kind="ref"`` loads ``oracle/_ref/libtdlb_ref.so``: the reference's own CPU
  ``ComputeUnit`` compiled in place from its sources (``oracle/Makefile``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, and only as the checker. Both libraries keep the
reference's data model: a ghosted (ghost = 1) AoS lattice
``Q[xg, yg, zg, 18]`` holding moments between steps, ``F[xg, yg, zg, 3]``,
``Nu[xg, yg, zg]``; ``index = i*(yg*zg) + j*zg + k`` (ComputeUnit.hpp:454-463).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "libtdlb_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libtdlb_ref.so")

MARKER_DTYPE = np.dtype(
    [
        ("i", np.int64), ("j", np.int64), ("k", np.int64),
        ("iCartFraction", np.float32), ("kCartFraction", np.float32),
        ("uDelta", np.float32), ("vDelta", np.float32), ("wDelta", np.float32),
        ("pad", np.float32),
    ]
)
assert MARKER_DTYPE.itemsize == 48


class _Flow(ctypes.Structure):
    _fields_ = [
        ("initialRho", ctypes.c_double), ("nu", ctypes.c_double), ("cs0", ctypes.c_double),
        ("g3", ctypes.c_double), ("alpha", ctypes.c_double), ("beta", ctypes.c_double),
        ("useLES", ctypes.c_int32), ("pad", ctypes.c_int32),
    ]


@dataclass
class Flow:
    """The FlowParams fields the time step reads (FlowParams.hpp:24-61)."""

    initialRho: float = 1.0
    nu: float = 0.0
    cs0: float = 0.1
    g3: float = 0.8
    alpha: float = 0.97
    beta: float = 1.9
    useLES: bool = True

    def c(self) -> _Flow:
        return _Flow(self.initialRho, self.nu, self.cs0, self.g3, self.alpha, self.beta, int(self.useLES), 0)


_LIBS: dict[str, ctypes.CDLL] = {}


def available(kind: str) -> bool:
    return os.path.exists(PORT_LIB if kind == "port" else REF_LIB)


def load(kind: str) -> ctypes.CDLL:
    if kind in _LIBS:
        return _LIBS[kind]
    path = PORT_LIB if kind == "port" else REF_LIB
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library {path} is not built (make -C oracle)")
    lib = ctypes.CDLL(path)
    p = "tdlbo_" if kind == "port" else "tdlbref_"
    vp, cl, cd, ci = ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_int
    sig = {
        "create": (vp, [ci, ci, cl, cl, cl, ctypes.POINTER(_Flow), ctypes.c_char_p]),
        "destroy": (None, [vp]), "size": (cl, [vp]), "even_step": (ci, [vp]),
        "set_even_step": (None, [vp, ci]), "set_nu": (None, [vp, cd]),
        "initialise": (None, [vp, cd]), "collision": (None, [vp]), "bounce_back": (None, [vp]),
        "streaming_push": (None, [vp]), "moments": (None, [vp]),
        "forcing": (None, [vp, vp, cl, cd, cd]), "step": (None, [vp, vp, cl, cd, cd]),
        "get_q": (None, [vp, vp]), "set_q": (None, [vp, vp]), "get_moments": (None, [vp, vp]), "get_f": (None, [vp, vp]),
        "set_f": (None, [vp, vp]), "get_nu": (None, [vp, vp]), "set_nu_field": (None, [vp, vp]),
        "kat_simple_stream": (ci, [ci, cl, cl, cl, vp]),
        "kat_esotwist": (ci, [cl, cl, cl, ci, ci, ci, vp]),
        "kat_esotwist_read": (ci, [cl, cl, cl, ci, vp]),
    }
    if kind == "port":
        sig["get_o"] = (None, [vp, vp])
        sig["transport"] = (None, [vp])
        sig["get_forcing_sums"] = (None, [vp, vp, cl])
        sig["set_threads"] = (None, [ci])
        sig["get_moments_range"] = (None, [vp, cl, cl, vp])
    else:
        sig["kat_simple_golden"] = (ci, [ci, vp])
        sig["checkpoint_write"] = (cl, [vp, ctypes.c_char_p, cl, ctypes.c_char_p, cl])
        sig["checkpoint_read"] = (ci, [vp, ctypes.c_char_p, ctypes.c_char_p])
        sig["calc_nu"] = (cd, [cd, cd, ci])
        sig["set_exclude"] = (None, [vp, vp, cl, ci])
        sig["save_plane_xz"] = (cl, [vp, cl, cl, ctypes.c_char_p, cl])
    for name, (res, args) in sig.items():
        fn = getattr(lib, p + name)
        fn.restype = res
        fn.argtypes = args
    lib._tdlb_prefix = p
    _LIBS[kind] = lib
    return lib


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


class CpuLattice:
    """One reference-style ComputeUnit on the CPU (``kind`` = "port" | "ref")."""

    def __init__(self, kind: str, x: int, y: int, z: int, flow: Flow, streaming: str = "Simple",
                 precision: int = 4, tmpdir: str = "/tmp"):
        self.kind = kind
        self.lib = load(kind)
        self.p = self.lib._tdlb_prefix
        self.x, self.y, self.z = x, y, z
        self.shape = (x + 2, y + 2, z + 2)
        self.flow = flow
        st = 0 if streaming == "Simple" else 1
        self._flow_c = flow.c()
        self.h = self._fn("create")(precision, st, x, y, z, ctypes.byref(self._flow_c), tmpdir.encode())
        if not self.h:
            raise ValueError("oracle create failed")

    def _fn(self, name):
        return getattr(self.lib, self.p + name)

    def close(self):
        if self.h:
            self._fn("destroy")(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass

    # --- the ComputeUnit virtuals, main.cpp order ---
    def initialise(self, rho: float):
        self._fn("initialise")(self.h, rho)

    def collision(self):
        self._fn("collision")(self.h)

    def bounce_back(self):
        self._fn("bounce_back")(self.h)

    def streaming_push(self):
        self._fn("streaming_push")(self.h)

    def moments(self):
        self._fn("moments")(self.h)

    def forcing(self, markers: np.ndarray, alpha: float, beta: float):
        m = np.ascontiguousarray(markers, dtype=MARKER_DTYPE)
        self._fn("forcing")(self.h, _ptr(m), len(m), alpha, beta)

    def step(self, markers: np.ndarray, alpha: float, beta: float):
        m = np.ascontiguousarray(markers, dtype=MARKER_DTYPE)
        self._fn("step")(self.h, _ptr(m), len(m), alpha, beta)

    @property
    def even_step(self) -> bool:
        return bool(self._fn("even_step")(self.h))

    @even_step.setter
    def even_step(self, v: bool):
        self._fn("set_even_step")(self.h, int(v))

    def set_nu(self, nu: float):
        self._fn("set_nu")(self.h, nu)

    # --- fields (float64 copies; float32 -> float64 is exact) ---
    def get_q(self) -> np.ndarray:
        out = np.empty(self.shape + (18,), np.float64)
        self._fn("get_q")(self.h, _ptr(out))
        return out

    def set_q(self, q: np.ndarray):
        a = np.ascontiguousarray(q, dtype=np.float64).reshape(self.shape + (18,))
        self._fn("set_q")(self.h, _ptr(a))

    def get_moments(self) -> np.ndarray:
        """Interior moments [x, y, z, 18] through the reference's read accessor."""
        out = np.empty((self.x, self.y, self.z, 18), np.float64)
        self._fn("get_moments")(self.h, _ptr(out))
        return out

    def get_moments_range(self, i0: int, i1: int) -> np.ndarray:
        """Interior moments of the slab i0 <= i < i1 [i1-i0, y, z, 18] (port only)."""
        out = np.empty((i1 - i0, self.y, self.z, 18), np.float64)
        self._fn("get_moments_range")(self.h, i0, i1, _ptr(out))
        return out

    def interior(self, a: np.ndarray) -> np.ndarray:
        return a[1:-1, 1:-1, 1:-1]

    def get_f(self) -> np.ndarray:
        out = np.empty(self.shape + (3,), np.float64)
        self._fn("get_f")(self.h, _ptr(out))
        return out

    def set_f(self, f: np.ndarray):
        a = np.ascontiguousarray(f, dtype=np.float64).reshape(self.shape + (3,))
        self._fn("set_f")(self.h, _ptr(a))

    def get_nu(self) -> np.ndarray:
        out = np.empty(self.shape, np.float64)
        self._fn("get_nu")(self.h, _ptr(out))
        return out

    def set_nu_field(self, nu: np.ndarray):
        a = np.ascontiguousarray(nu, dtype=np.float64).reshape(self.shape)
        self._fn("set_nu_field")(self.h, _ptr(a))

    def transport(self):
        """Identity-collision step: Simple push, or Esotwist read+write+flip (port only)."""
        self._fn("transport")(self.h)

    def get_forcing_sums(self, n: int) -> np.ndarray:
        """Per-marker spread sums [n, 3] of the last forcing() (port only)."""
        out = np.empty((n, 3), np.float64)
        self._fn("get_forcing_sums")(self.h, _ptr(out), n)
        return out

    def checkpoint_write(self, unit: str, step: int) -> str:
        """The reference's own checkpoint_write (ref only); returns its directory."""
        buf = ctypes.create_string_buffer(4096)
        n = self._fn("checkpoint_write")(self.h, unit.encode(), step, buf, len(buf))
        if n <= 0:
            raise RuntimeError("reference checkpoint_write failed")
        return buf.value.decode()

    def checkpoint_read(self, directory: str, unit: str):
        """The reference's own checkpoint_read (ref only)."""
        if self._fn("checkpoint_read")(self.h, directory.encode(), unit.encode()) != 0:
            raise RuntimeError("reference checkpoint_read failed")

    def set_exclude(self, markers: np.ndarray, exclude: bool = True):
        """The reference's setOutputExcludePoints / unset (ref only)."""
        m = np.ascontiguousarray(markers)
        self._fn("set_exclude")(self.h, _ptr(m), len(m), 1 if exclude else 0)

    def save_plane_xz(self, j: int, step: int) -> str:
        """The reference's savePlaneXZ<float, 4> (ref only); returns its directory."""
        buf = ctypes.create_string_buffer(4096)
        if self._fn("save_plane_xz")(self.h, j, step, buf, len(buf)) <= 0:
            raise RuntimeError("reference savePlaneXZ failed")
        return buf.value.decode()

    def get_o(self) -> np.ndarray:
        """Cells the last forcing() touched (port only; the reference resets O)."""
        out = np.empty(self.shape, np.uint8)
        self._fn("get_o")(self.h, _ptr(out))
        return out


def kat_simple_stream(kind: str, push: bool, x: int, y: int, z: int) -> np.ndarray:
    lib = load(kind)
    out = np.zeros((x + 2) * (y + 2) * (z + 2) * 18, np.uint64)
    rc = getattr(lib, lib._tdlb_prefix + "kat_simple_stream")(int(push), x, y, z, _ptr(out))
    if rc:
        raise ValueError(f"kat_simple_stream rc={rc}")
    return out.reshape(x + 2, y + 2, z + 2, 18)


def kat_simple_golden(push: bool) -> np.ndarray:
    lib = load("ref")
    out = np.zeros(5 * 5 * 5 * 18, np.uint64)
    rc = lib.tdlbref_kat_simple_golden(int(push), _ptr(out))
    if rc:
        raise ValueError(f"kat_simple_golden rc={rc}")
    return out.reshape(5, 5, 5, 18)


def kat_esotwist(kind: str, x: int, y: int, z: int, start_even: bool, nsteps: int, moments_map: bool) -> np.ndarray:
    lib = load(kind)
    out = np.zeros((x + 2) * (y + 2) * (z + 2) * 18, np.uint64)
    rc = getattr(lib, lib._tdlb_prefix + "kat_esotwist")(x, y, z, int(start_even), nsteps, int(moments_map), _ptr(out))
    if rc:
        raise ValueError(f"kat_esotwist rc={rc}")
    return out.reshape(x + 2, y + 2, z + 2, 18)


def kat_esotwist_read(kind: str, x: int, y: int, z: int, even: bool) -> np.ndarray:
    lib = load(kind)
    out = np.zeros(x * y * z * 18, np.uint64)
    rc = getattr(lib, lib._tdlb_prefix + "kat_esotwist_read")(x, y, z, int(even), _ptr(out))
    if rc:
        raise ValueError(f"kat_esotwist_read rc={rc}")
    return out.reshape(x, y, z, 18)


def coded_fill(x: int, y: int, z: int) -> np.ndarray:
    """The integer coding of tests/Params/ParamsCommon.hpp:168-206 (offset 0):
    Q(i,j,k,l) = ((i*100+j)*100+k)*100+l over the ghosted grid."""
    i, j, k, l = np.meshgrid(np.arange(x + 2), np.arange(y + 2), np.arange(z + 2), np.arange(18), indexing="ij")
    return (((i * 100 + j) * 100 + k) * 100 + l).astype(np.uint64)


class _RushtonSpec(ctypes.Structure):
    """Same layout as tdlb_rushton (include/tdlb_b200.h)."""

    _fields_ = [
        ("x", ctypes.c_int64), ("y", ctypes.c_int64), ("z", ctypes.c_int64),
        ("tank_diameter", ctypes.c_double), ("impeller_diameter", ctypes.c_double),
        ("clearance", ctypes.c_double), ("blade_height", ctypes.c_double), ("disk_thickness", ctypes.c_double),
        ("n_blades", ctypes.c_int32), ("n_baffles", ctypes.c_int32),
        ("baffle_width", ctypes.c_double), ("wall_inset", ctypes.c_double), ("tip_speed", ctypes.c_double),
        ("startup_steps", ctypes.c_int64),
    ]


class RefRushton:
    """The project's Rushton-turbine marker generator as compiled into the
    reference harness (oracle/_ref/libtdlb_ref.so carries
    tdlbcpp_b200/csrc/geometry.cpp), so that a process timing the reference
    builds its marker lists without loading the B200 library. Same methods
    and results as tdlbcpp_b200.RushtonTurbine."""

    def __init__(self, x: int, y: int, z: int, tip_speed: float = 0.1, startup_steps: int = 0):
        lib = load("ref")
        if not hasattr(lib, "_rushton_bound"):
            sz, vp = ctypes.c_size_t, ctypes.c_void_p
            sp = ctypes.POINTER(_RushtonSpec)
            for name, extra in (("fixed", []), ("rotating_nonupdating", [ctypes.c_double]),
                                ("rotating", [ctypes.c_double, ctypes.c_double])):
                fn = getattr(lib, "tdlb_rushton_" + name)
                fn.restype = ctypes.c_int
                fn.argtypes = [sp, *extra, vp, sz, ctypes.POINTER(sz)]
            lib.tdlb_rushton_impeller_increment.restype = ctypes.c_double
            lib.tdlb_rushton_impeller_increment.argtypes = [sp, ctypes.c_uint64]
            lib.tdlb_rushton_blade_outer_radius.restype = ctypes.c_int
            lib.tdlb_rushton_blade_outer_radius.argtypes = [sp]
            lib._rushton_bound = True
        self.lib = lib
        self.spec = _RushtonSpec()
        self.spec.x, self.spec.y, self.spec.z = x, y, z
        self.spec.tip_speed = tip_speed
        self.spec.startup_steps = startup_steps

    def _gen(self, name, *args) -> np.ndarray:
        fn = getattr(self.lib, "tdlb_rushton_" + name)
        n = ctypes.c_size_t()
        if fn(ctypes.byref(self.spec), *args, None, 0, ctypes.byref(n)):
            raise ValueError(f"tdlb_rushton_{name} failed")
        out = np.zeros(n.value, MARKER_DTYPE)
        if fn(ctypes.byref(self.spec), *args, _ptr(out), n.value, ctypes.byref(n)):
            raise ValueError(f"tdlb_rushton_{name} failed")
        return out

    def fixed(self) -> np.ndarray:
        return self._gen("fixed")

    def rotating_nonupdating(self, delta_angle: float) -> np.ndarray:
        return self._gen("rotating_nonupdating", ctypes.c_double(delta_angle))

    def rotating(self, angle: float, delta_angle: float) -> np.ndarray:
        return self._gen("rotating", ctypes.c_double(angle), ctypes.c_double(delta_angle))

    def increment(self, step: int) -> float:
        return self.lib.tdlb_rushton_impeller_increment(ctypes.byref(self.spec), step)

    def blade_outer_radius(self) -> int:
        return self.lib.tdlb_rushton_blade_outer_radius(ctypes.byref(self.spec))

    def forcing_list(self, angle: float, delta_angle: float, nonupdating_delta: float = None) -> np.ndarray:
        """fixed + rotating-non-updating + rotating, the order main.cpp:301-303 builds."""
        nd = delta_angle if nonupdating_delta is None else nonupdating_delta
        return np.concatenate([self.fixed(), self.rotating_nonupdating(nd), self.rotating(angle, delta_angle)])


def ref_nu(re: float, tip_speed: float, blade_outer_radius: int) -> float:
    """The reference's own FlowParams::calcNuAndRe_m (FlowParams.hpp:65-70)."""
    return float(load("ref").tdlbref_calc_nu(re, tip_speed, blade_outer_radius))


def reference_root() -> str:
    """The reference checkout the oracle compiles from (oracle/Makefile's
    REF_ROOT: the TDLB_REFERENCE environment variable or its default)."""
    import subprocess
    env = {k: v for k, v in os.environ.items() if k not in ("MAKEFLAGS", "MAKELEVEL", "MFLAGS")}
    r = subprocess.run(["make", "-s", "--no-print-directory", "-C", HERE, "print-ref-root"], capture_output=True,
                       text=True, check=True, env=env)
    return r.stdout.strip()


def ref_read_input(path: str) -> dict:
    """What a ComputeUnit built by main.cpp from the input file at `path`
    holds, read by the reference's own GridParams / FlowParams parsers
    (tdlbref_read_input)."""
    lib = load("ref")
    fn = lib.tdlbref_read_input
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(_Flow), ctypes.c_void_p]
    xyz = np.zeros(3, np.int64)
    ms = np.zeros(1, np.int64)
    st = np.zeros(1, np.int32)
    f = _Flow()
    if fn(path.encode(), _ptr(xyz), _ptr(ms), ctypes.byref(f), _ptr(st)):
        raise ValueError(f"the reference could not read {path}")
    return {"x": int(xyz[0]), "y": int(xyz[1]), "z": int(xyz[2]), "multiStep": int(ms[0]),
            "initialRho": f.initialRho, "nu": f.nu, "cs0": f.cs0, "g3": f.g3, "alpha": f.alpha, "beta": f.beta,
            "useLES": bool(f.useLES), "streaming": "Simple" if st[0] == 0 else "Esotwist"}
