"""B200-native lattice Boltzmann time step with tdLBCpp's ComputeUnit interface.

The compute path is the in-tree CUDA library ``libtdlb_b200.so`` (sm_100a),
reached through its C ABI (``include/tdlb_b200.h``) with ctypes. This module
is the host-side mirror of the reference's ``ComputeUnitBase`` virtuals
(tdlbcpp/src/ComputeUnit.h:86-201) for Python callers; C++ callers use
``include/tdlb_compute_unit_b200.hpp``.

There is no CPU fallback: importing works anywhere, but creating a
``ComputeUnit`` without the built library or without an sm_100 GPU raises.
"""
from __future__ import annotations

import ctypes
import json
import os
from typing import Optional

import numpy as np

__all__ = [
    "ComputeUnit", "Batch", "Server", "TdlbError", "MARKER_DTYPE", "library_path", "load_library", "make_config",
    "STREAMING_SIMPLE", "STREAMING_ESOTWIST",
]

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
_LIB_NAME = "libtdlb_b200.so"

STREAMING_SIMPLE = 0
STREAMING_ESOTWIST = 1
STORAGE_FP32 = 0
STORAGE_FP16 = 1
STORAGE_BF16 = 2

# Lattice vectors of population slots Q01..Q18 (tdlbcpp/src/Header.h:70-100);
# opposite(d) = d ^ 1.
CX = (1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0)
CY = (0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1)
CZ = (0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1)

# tdlb_marker (include/tdlb_b200.h): the PosPolar fields forcing() reads.
MARKER_DTYPE = np.dtype(
    [
        ("i", np.int64), ("j", np.int64), ("k", np.int64),
        ("iCartFraction", np.float32), ("kCartFraction", np.float32),
        ("uDelta", np.float32), ("vDelta", np.float32), ("wDelta", np.float32),
        ("pad", np.float32),
    ]
)
assert MARKER_DTYPE.itemsize == 48

# tdlb_disk_grid4 / tdlb_disk_grid3: the reference's tDiskGrid<float, 4 / 3>
# plane-dump records (Output.hpp:22-26).
DISK_GRID4_DTYPE = np.dtype([("iGrid", np.uint16), ("jGrid", np.uint16), ("kGrid", np.uint16), ("pad", np.uint16),
                             ("q", np.float32, 4)])
DISK_GRID3_DTYPE = np.dtype([("iGrid", np.uint16), ("jGrid", np.uint16), ("kGrid", np.uint16), ("pad", np.uint16),
                             ("q", np.float32, 3)])
assert DISK_GRID4_DTYPE.itemsize == 24 and DISK_GRID3_DTYPE.itemsize == 20

_ERRORS = {
    -1: "TDLB_EINVAL", -2: "TDLB_ECUDA", -3: "TDLB_ENOMEM", -4: "TDLB_EIO", -5: "TDLB_ESTATE", -6: "TDLB_EJSON",
}


class TdlbError(RuntimeError):
    """A C-ABI call returned a non-zero status (the reference would have
    called exit(1) or thrown std::runtime_error)."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{_ERRORS.get(code, code)}: {message}")
        self.code = code


class Config(ctypes.Structure):
    """tdlb_config: the GridParams / FlowParams fields the step reads."""

    _fields_ = [
        ("x", ctypes.c_int64), ("y", ctypes.c_int64), ("z", ctypes.c_int64),
        ("streaming", ctypes.c_int32), ("storage", ctypes.c_int32),
        ("initialRho", ctypes.c_double), ("nu", ctypes.c_double), ("cs0", ctypes.c_double),
        ("g3", ctypes.c_double), ("alpha", ctypes.c_double), ("beta", ctypes.c_double),
        ("useLES", ctypes.c_int32), ("reserved", ctypes.c_int32),
    ]


class Rushton(ctypes.Structure):
    """tdlb_rushton: the project's Rushton-turbine tank spec (zero = default)."""

    _fields_ = [
        ("x", ctypes.c_int64), ("y", ctypes.c_int64), ("z", ctypes.c_int64),
        ("tank_diameter", ctypes.c_double), ("impeller_diameter", ctypes.c_double),
        ("clearance", ctypes.c_double), ("blade_height", ctypes.c_double), ("disk_thickness", ctypes.c_double),
        ("n_blades", ctypes.c_int32), ("n_baffles", ctypes.c_int32),
        ("baffle_width", ctypes.c_double), ("wall_inset", ctypes.c_double), ("tip_speed", ctypes.c_double),
        ("startup_steps", ctypes.c_int64),
    ]


class Request(ctypes.Structure):
    """tdlb_request: one tank solve submitted to a Server."""

    _fields_ = [
        ("id", ctypes.c_int64), ("x", ctypes.c_int64), ("y", ctypes.c_int64), ("z", ctypes.c_int64),
        ("tip_speed", ctypes.c_double), ("reynolds", ctypes.c_double), ("steps", ctypes.c_int64),
        ("storage", ctypes.c_int32), ("streaming", ctypes.c_int32), ("les", ctypes.c_int32), ("pad", ctypes.c_int32),
        ("out_rho", ctypes.c_void_p), ("out_ux", ctypes.c_void_p), ("out_uy", ctypes.c_void_p),
        ("out_uz", ctypes.c_void_p),
    ]


class Result(ctypes.Structure):
    """tdlb_result: a finished request's timing and FP64 diagnostics."""

    _fields_ = [
        ("id", ctypes.c_int64), ("status", ctypes.c_int32), ("pad", ctypes.c_int32),
        ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double),
        ("cells", ctypes.c_int64), ("steps", ctypes.c_int64), ("mass", ctypes.c_double),
        ("momentum", ctypes.c_double * 3), ("force", ctypes.c_double * 3), ("torque", ctypes.c_double),
        ("power_number", ctypes.c_double),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("queued", ctypes.c_int64),
        ("active", ctypes.c_int64), ("admitted", ctypes.c_int64), ("chunks", ctypes.c_int64),
        ("bytes_in_use", ctypes.c_int64), ("lattice_updates", ctypes.c_double), ("busy_s", ctypes.c_double),
        ("elapsed_s", ctypes.c_double),
    ]


def make_config(**fields) -> Config:
    """A tdlb_config from keyword fields. Unnamed fields: cs0 0.12, g3 0.8,
    alpha 0.97, beta 1.9, useLES off (the reference's FlowParams defaults,
    FlowParams.hpp:32-59) and initialRho 1 (the reference's is 8). ``streaming``
    may be "Simple" or "Esotwist", ``storage`` "fp32", "fp16" or "bf16"."""
    cfg = Config()
    cfg.streaming = STREAMING_SIMPLE
    cfg.initialRho, cfg.cs0, cfg.g3, cfg.alpha, cfg.beta, cfg.useLES = 1.0, 0.12, 0.8, 0.97, 1.9, 0
    for key, val in fields.items():
        if key == "streaming" and isinstance(val, str):
            val = STREAMING_SIMPLE if val == "Simple" else STREAMING_ESOTWIST
        if key == "storage" and isinstance(val, str):
            val = {"fp32": STORAGE_FP32, "fp16": STORAGE_FP16, "bf16": STORAGE_BF16}[val.lower()]
        setattr(cfg, key, val)
    return cfg


def config_from_json(params_json: str) -> Config:
    """The tdlb_config tdlb_create builds from a reference input file's text
    (host only; raises TdlbError on a malformed or incomplete file)."""
    lib = load_library()
    cfg = Config()
    rc = lib.tdlb_config_from_json(params_json.encode(), ctypes.byref(cfg))
    if rc:
        raise TdlbError(rc, lib.tdlb_last_error(None).decode())
    return cfg


def library_path() -> str:
    return os.path.join(HERE, _LIB_NAME)


_lib: Optional[ctypes.CDLL] = None


def load_library() -> ctypes.CDLL:
    """Load the in-tree CUDA library; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `make -C tdlbcpp_b200` (there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    H, vp, i32, f32, sz = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_size_t
    sigs = {
        "tdlb_create": (i32, [ctypes.c_char_p, i32, ctypes.POINTER(H)]),
        "tdlb_create_config": (i32, [ctypes.POINTER(Config), i32, ctypes.POINTER(H)]),
        "tdlb_config_from_json": (i32, [ctypes.c_char_p, ctypes.POINTER(Config)]),
        "tdlb_destroy": (i32, [H]),
        "tdlb_last_error": (ctypes.c_char_p, [H]),
        "tdlb_initialise": (i32, [H, f32]),
        "tdlb_forcing": (i32, [H, vp, sz, f32, f32]),
        "tdlb_set_markers": (i32, [H, vp, sz]),
        "tdlb_forcing_resident": (i32, [H, f32, f32]),
        "tdlb_collision": (i32, [H]),
        "tdlb_bounce_back": (i32, [H]),
        "tdlb_streaming_push": (i32, [H]),
        "tdlb_moments": (i32, [H]),
        "tdlb_step": (i32, [H, f32, f32]),
        "tdlb_read_moments": (i32, [H, vp]),
        "tdlb_read_velocity_density": (i32, [H, vp, vp, vp, vp]),
        "tdlb_read_force": (i32, [H, vp]),
        "tdlb_read_nu": (i32, [H, vp]),
        "tdlb_read_touched": (i32, [H, vp]),
        "tdlb_get_dims": (i32, [H, vp, vp, vp]),
        "tdlb_get_even_step": (i32, [H, vp]),
        "tdlb_synchronize": (i32, [H]),
        "tdlb_debug_get_state": (i32, [H, vp]),
        "tdlb_debug_set_state": (i32, [H, vp, i32]),
        "tdlb_debug_transport": (i32, [H]),
        "tdlb_rushton_fixed": (i32, [ctypes.POINTER(Rushton), vp, sz, ctypes.POINTER(sz)]),
        "tdlb_rushton_rotating_nonupdating": (i32, [ctypes.POINTER(Rushton), ctypes.c_double, vp, sz, ctypes.POINTER(sz)]),
        "tdlb_rushton_rotating": (i32, [ctypes.POINTER(Rushton), ctypes.c_double, ctypes.c_double, vp, sz, ctypes.POINTER(sz)]),
        "tdlb_rushton_impeller_increment": (ctypes.c_double, [ctypes.POINTER(Rushton), ctypes.c_uint64]),
        "tdlb_rushton_blade_outer_radius": (i32, [ctypes.POINTER(Rushton)]),
        "tdlb_schedule_levels": (i32, [vp, sz, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, vp, vp]),
        "tdlb_attach_rushton": (i32, [H, ctypes.POINTER(Rushton), ctypes.c_double, ctypes.c_double, ctypes.c_double]),
        "tdlb_rotate_impeller": (i32, [H, ctypes.c_double, ctypes.c_double]),
        "tdlb_read_markers": (i32, [H, vp, sz, ctypes.POINTER(sz)]),
        "tdlb_set_rotating_markers": (i32, [H, vp, sz]),
        "tdlb_impeller_load": (i32, [H, vp]),
        "tdlb_impeller_load_noalloc": (i32, [H, vp]),
        "tdlb_impeller_load_async": (i32, [H, vp]),
        "tdlb_get_stream": (i32, [H, ctypes.POINTER(ctypes.c_void_p)]),
        "tdlb_set_cells_per_thread": (i32, [H, i32]),
        "tdlb_set_l2_prefetch": (i32, [H, i32]),
        "tdlb_set_residual_box": (i32, [H] + [ctypes.c_int64] * 6),
        "tdlb_get_residual_box": (i32, [H, vp]),
        "tdlb_set_overlap": (i32, [H, i32]),
        "tdlb_join": (i32, [H]),
        "tdlb_read_zone": (i32, [H, vp]),
        "tdlb_set_kernel_timing": (i32, [H, i32]),
        "tdlb_kernel_launches": (i32, [H, ctypes.POINTER(ctypes.c_int64)]),
        "tdlb_kernel_time": (i32, [H, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]),
        "tdlb_reduce_fp64": (i32, [H, vp]),
        "tdlb_checkpoint_write": (i32, [H, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p]),
        "tdlb_checkpoint_read": (i32, [H, ctypes.c_char_p, ctypes.c_char_p]),
        "tdlb_set_output_exclude": (i32, [H, vp, sz, i32]),
        "tdlb_double_resolution": (i32, [H]),
        "tdlb_vorticity_xz": (i32, [H, ctypes.c_int64, vp]),
        "tdlb_vorticity_xy": (i32, [H, ctypes.c_int64, vp]),
        "tdlb_plane_xz": (i32, [H, ctypes.c_int64, vp, sz, ctypes.POINTER(sz), vp, sz, ctypes.POINTER(sz)]),
        "tdlb_batch_create": (i32, [ctypes.POINTER(Config), i32, i32, ctypes.POINTER(H)]),
        "tdlb_batch_destroy": (i32, [H]),
        "tdlb_batch_last_error": (ctypes.c_char_p, [H]),
        "tdlb_batch_size": (i32, [H, ctypes.POINTER(i32)]),
        "tdlb_batch_tank": (i32, [H, i32, ctypes.POINTER(H)]),
        "tdlb_batch_add": (i32, [H, ctypes.POINTER(Config), ctypes.POINTER(i32)]),
        "tdlb_batch_adopt": (i32, [H, H, ctypes.POINTER(i32)]),
        "tdlb_batch_detach": (i32, [H, i32, ctypes.POINTER(H)]),
        "tdlb_batch_remove": (i32, [H, i32]),
        "tdlb_batch_set_shape": (i32, [H, i32, i32, i32]),
        "tdlb_batch_get_shape": (i32, [H, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i32)]),
        "tdlb_batch_autotune": (i32, [H, i32, ctypes.POINTER(ctypes.c_double)]),
        "tdlb_batch_run": (i32, [H, i32, f32, f32]),
        "tdlb_batch_run_eager": (i32, [H, i32, f32, f32]),
        "tdlb_batch_synchronize": (i32, [H]),
        "tdlb_batch_create_empty": (i32, [i32, i32, i32, ctypes.POINTER(H)]),
        "tdlb_lattice_bytes": (i32, [ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_int64)]),
        "tdlb_server_create": (i32, [i32, ctypes.c_int64, i32, i32, ctypes.POINTER(H)]),
        "tdlb_server_destroy": (i32, [H]),
        "tdlb_server_last_error": (ctypes.c_char_p, [H]),
        "tdlb_server_submit": (i32, [H, ctypes.POINTER(Request)]),
        "tdlb_server_poll": (i32, [H, ctypes.POINTER(Result), i32, ctypes.POINTER(i32)]),
        "tdlb_server_wait_idle": (i32, [H, ctypes.c_double]),
        "tdlb_server_get_stats": (i32, [H, ctypes.POINTER(ServerStats)]),
        "tdlb_batch_kernel_launches": (i32, [H, ctypes.POINTER(ctypes.c_longlong)]),
        "tdlb_batch_get_stream": (i32, [H, ctypes.POINTER(ctypes.c_void_p)]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _p(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def as_markers(markers) -> np.ndarray:
    m = np.ascontiguousarray(markers)
    if m.dtype != MARKER_DTYPE:
        out = np.zeros(len(m), MARKER_DTYPE)
        for name in MARKER_DTYPE.names:
            if name in (m.dtype.names or ()):
                out[name] = m[name]
        m = out
    return m


class ComputeUnit:
    """One lattice on one GPU, driven like the reference's ComputeUnitBase.

    Construct from the reference's input JSON (a path, a JSON string or a
    dict) or from keyword fields of ``tdlb_config``. The reference call
    sequence per step is kept: ``collision(); bounceBackBoundary();
    streamingPush(); moments(); forcing(markers, alpha, beta)``.
    """

    def __init__(self, params=None, device: int = 0, **config):
        self.lib = load_library()
        h = ctypes.c_void_p()
        if params is not None:
            if isinstance(params, dict):
                text = json.dumps(params)
            elif isinstance(params, str) and params.lstrip().startswith("{"):
                text = params
            else:
                with open(params) as f:
                    text = f.read()
            rc = self.lib.tdlb_create(text.encode(), device, ctypes.byref(h))
        else:
            rc = self.lib.tdlb_create_config(ctypes.byref(make_config(**config)), device, ctypes.byref(h))
        if rc != 0:
            raise TdlbError(rc, self.lib.tdlb_last_error(None).decode())
        self._attach(h, owned=True)

    @classmethod
    def _borrowed(cls, lib: ctypes.CDLL, h: ctypes.c_void_p) -> "ComputeUnit":
        """A view of a tank that a Batch owns (closing it does nothing)."""
        cu = cls.__new__(cls)
        cu.lib = lib
        cu._attach(h, owned=False)
        return cu

    def _attach(self, h: ctypes.c_void_p, owned: bool):
        self.h = h
        self._owned = owned
        x, y, z = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.tdlb_get_dims(self.h, ctypes.byref(x), ctypes.byref(y), ctypes.byref(z)))
        self.x, self.y, self.z = x.value, y.value, z.value

    # ---- lifecycle ----
    def _check(self, rc: int):
        if rc != 0:
            raise TdlbError(rc, self.lib.tdlb_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "_owned", True):
                self.lib.tdlb_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    @property
    def ncell(self) -> int:
        return self.x * self.y * self.z

    # ---- ComputeUnitBase virtuals (ComputeUnit.h:110-200) ----
    def initialise(self, rho: float):
        self._check(self.lib.tdlb_initialise(self.h, rho))

    def forcing(self, markers, alpha: float, beta: float):
        m = as_markers(markers)
        self._check(self.lib.tdlb_forcing(self.h, _p(m), len(m), alpha, beta))

    def set_markers(self, markers):
        m = as_markers(markers)
        self._check(self.lib.tdlb_set_markers(self.h, _p(m), len(m)))

    def forcing_resident(self, alpha: float, beta: float):
        self._check(self.lib.tdlb_forcing_resident(self.h, alpha, beta))

    def collision(self):
        self._check(self.lib.tdlb_collision(self.h))

    def bounceBackBoundary(self):
        self._check(self.lib.tdlb_bounce_back(self.h))

    def streamingPush(self):
        self._check(self.lib.tdlb_streaming_push(self.h))

    def moments(self):
        self._check(self.lib.tdlb_moments(self.h))

    def step(self, alpha: float, beta: float):
        self._check(self.lib.tdlb_step(self.h, alpha, beta))

    def synchronize(self):
        self._check(self.lib.tdlb_synchronize(self.h))

    @property
    def evenStep(self) -> bool:
        e = ctypes.c_int()
        self._check(self.lib.tdlb_get_even_step(self.h, ctypes.byref(e)))
        return bool(e.value)

    # ---- resident impeller (device-side rotation) ----
    def attach_rushton(self, turbine: "RushtonTurbine", nonupdating_delta: float, angle: float, delta: float):
        self._check(self.lib.tdlb_attach_rushton(self.h, ctypes.byref(turbine.spec), nonupdating_delta, angle, delta))

    def rotate_impeller(self, angle: float, delta: float):
        self._check(self.lib.tdlb_rotate_impeller(self.h, angle, delta))

    def set_rotating_markers(self, markers):
        m = as_markers(markers)
        self._check(self.lib.tdlb_set_rotating_markers(self.h, _p(m), len(m)))

    def impeller_load(self, out: np.ndarray = None) -> np.ndarray:
        """FP64 (Fx, Fy, Fz, torque_j, n_markers) on the attached impeller."""
        if out is None:
            out = np.zeros(5, np.float64)
        self._check(self.lib.tdlb_impeller_load(self.h, _p(out)))
        return out

    def reduce_fp64(self) -> np.ndarray:
        """FP64 (mass, momentum x, y, z) over all interior cells."""
        out = np.zeros(4, np.float64)
        self._check(self.lib.tdlb_reduce_fp64(self.h, _p(out)))
        return out

    # ---- checkpoint (ComputeUnit.hpp:318-439) ----
    def checkpoint_write(self, directory: str, unit_name: str, params=None):
        """Q/F/Nu + AllParams JSON in the reference's layout under `directory`.
        `params`: the run's params (dict or JSON text), e.g. its RunningParams."""
        text = None if params is None else (params if isinstance(params, str) else json.dumps(params))
        self._check(self.lib.tdlb_checkpoint_write(self.h, directory.encode(), unit_name.encode(),
                                                   None if text is None else text.encode()))

    def checkpoint_read(self, directory: str, unit_name: str):
        self._check(self.lib.tdlb_checkpoint_read(self.h, directory.encode(), unit_name.encode()))

    def doubleResolutionFullCU(self):
        """Double x, y, z on the device (ComputeUnit.hpp:258-316); set the
        geometry of the new size afterwards."""
        self._check(self.lib.tdlb_double_resolution(self.h))
        x, y, z = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.tdlb_get_dims(self.h, ctypes.byref(x), ctypes.byref(y), ctypes.byref(z)))
        self.x, self.y, self.z = x.value, y.value, z.value

    # ---- output (ComputeUnitOutput.hpp) ----
    def set_output_exclude(self, markers, exclude: bool = True):
        m = as_markers(markers)
        self._check(self.lib.tdlb_set_output_exclude(self.h, _p(m), len(m), 1 if exclude else 0))

    def vorticity_xz(self, j: int) -> np.ndarray:
        """log |curl u|^2 on the plane j, [x, z]; -1 at excluded points."""
        out = np.empty((self.x, self.z), np.float32)
        self._check(self.lib.tdlb_vorticity_xz(self.h, j, _p(out)))
        return out

    def vorticity_xy(self, k: int) -> np.ndarray:
        """log |curl u|^2 on the plane k, [y, x] (the reference's picture order)."""
        out = np.empty((self.y, self.x), np.float32)
        self._check(self.lib.tdlb_vorticity_xy(self.h, k, _p(out)))
        return out

    def plane_xz(self, j: int):
        """savePlaneXZ<float, 4> records: (moments of non-excluded cells, F where non-zero)."""
        nq, nf = ctypes.c_size_t(), ctypes.c_size_t()
        self._check(self.lib.tdlb_plane_xz(self.h, j, None, 0, ctypes.byref(nq), None, 0, ctypes.byref(nf)))
        q = np.zeros(nq.value, DISK_GRID4_DTYPE)
        f = np.zeros(nf.value, DISK_GRID3_DTYPE)
        self._check(self.lib.tdlb_plane_xz(self.h, j, _p(q), len(q), ctypes.byref(nq), _p(f), len(f), ctypes.byref(nf)))
        return q, f

    def set_cells_per_thread(self, v: int):
        """Step-kernel variant (1, 2 or 4 cells per thread)."""
        self._check(self.lib.tdlb_set_cells_per_thread(self.h, v))

    def set_l2_prefetch(self, on: bool):
        """Step kernels' L2 prefetch one wave ahead (on by default; results identical)."""
        self._check(self.lib.tdlb_set_l2_prefetch(self.h, 1 if on else 0))

    def set_residual_box(self, i0: int, i1: int, j0: int, j1: int, k0: int, k1: int):
        """16-bit storage: keep the locations of the box [i0,i1) x [j0,j1) x [k0,k1)
        exact (an empty box removes it; tdlb_set_residual_box)."""
        self._check(self.lib.tdlb_set_residual_box(self.h, i0, i1, j0, j1, k0, k1))

    def residual_box(self):
        """(i0, i1, j0, j1, k0, k1) of the residual box, all zero without one."""
        out = np.zeros(6, np.int64)
        self._check(self.lib.tdlb_get_residual_box(self.h, _p(out)))
        return tuple(int(v) for v in out)

    def set_overlap(self, mode):
        """Split steps: the outer cells of a step run while the previous
        forcing pass is in flight; results are identical. False/0 (default):
        off; True/1: when the inner chunks hold at most 60 % of the lattice;
        "always"/2: whenever the markers are resident."""
        m = 2 if mode == "always" else int(bool(mode)) if isinstance(mode, bool) else int(mode)
        self._check(self.lib.tdlb_set_overlap(self.h, m))

    def join(self):
        """Order this unit's stream after every queued step and forcing pass
        (no host wait): call before recording an event on `stream`."""
        self._check(self.lib.tdlb_join(self.h))

    def read_zone(self) -> np.ndarray:
        """Per-cell flags of the split-step inner chunks."""
        out = np.empty((self.x, self.y, self.z), np.uint8)
        self._check(self.lib.tdlb_read_zone(self.h, _p(out)))
        return out

    def set_kernel_timing(self, on: bool):
        """Bracket every step-kernel launch with CUDA events on its stream."""
        self._check(self.lib.tdlb_set_kernel_timing(self.h, 1 if on else 0))

    def kernel_time(self):
        """(summed step-kernel ms, launches) since the last call; waits for the device."""
        ms, n = ctypes.c_double(), ctypes.c_int64()
        self._check(self.lib.tdlb_kernel_time(self.h, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def kernel_launches(self) -> int:
        """Kernels the step loop has queued so far."""
        n = ctypes.c_int64()
        self._check(self.lib.tdlb_kernel_launches(self.h, ctypes.byref(n)))
        return n.value

    def impeller_load_async(self, ptr: int):
        """Queue the impeller load and its copy into 5 doubles at `ptr`
        (pinned host or device memory) on this unit's stream; no wait."""
        self._check(self.lib.tdlb_impeller_load_async(self.h, ctypes.c_void_p(ptr)))

    def impeller_load_noalloc(self, device_ptr: int):
        """Allocation-free impeller load into a caller-owned device buffer of
        5 doubles (queued on this unit's stream; not synchronised)."""
        self._check(self.lib.tdlb_impeller_load_noalloc(self.h, ctypes.c_void_p(device_ptr)))

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.lib.tdlb_get_stream(self.h, ctypes.byref(s)))
        return s.value or 0

    def read_markers(self) -> np.ndarray:
        n = ctypes.c_size_t()
        self._check(self.lib.tdlb_read_markers(self.h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, MARKER_DTYPE)
        self._check(self.lib.tdlb_read_markers(self.h, _p(out), n.value, ctypes.byref(n)))
        return out

    # ---- field read-back (interior cells, (i, j, k) order) ----
    def read_moments(self) -> np.ndarray:
        out = np.empty((self.x, self.y, self.z, 18), np.float32)
        self._check(self.lib.tdlb_read_moments(self.h, _p(out)))
        return out

    def read_velocity_density(self):
        shape = (self.x, self.y, self.z)
        rho, ux, uy, uz = (np.empty(shape, np.float32) for _ in range(4))
        self._check(self.lib.tdlb_read_velocity_density(self.h, _p(rho), _p(ux), _p(uy), _p(uz)))
        return rho, np.stack([ux, uy, uz], axis=-1)

    def read_force(self) -> np.ndarray:
        out = np.empty((self.x, self.y, self.z, 3), np.float32)
        self._check(self.lib.tdlb_read_force(self.h, _p(out)))
        return out

    def read_nu(self) -> np.ndarray:
        out = np.empty((self.x, self.y, self.z), np.float32)
        self._check(self.lib.tdlb_read_nu(self.h, _p(out)))
        return out

    def read_touched(self) -> np.ndarray:
        out = np.empty((self.x, self.y, self.z), np.uint8)
        self._check(self.lib.tdlb_read_touched(self.h, _p(out)))
        return out

    # ---- known-answer-test support ----
    def debug_get_state(self) -> np.ndarray:
        out = np.empty((self.x, self.y, self.z, 18), np.float32)
        self._check(self.lib.tdlb_debug_get_state(self.h, _p(out)))
        return out

    def debug_set_state(self, q: np.ndarray, holds_moments: bool):
        a = np.ascontiguousarray(q, dtype=np.float32).reshape(self.x, self.y, self.z, 18)
        self._check(self.lib.tdlb_debug_set_state(self.h, _p(a), int(holds_moments)))

    def debug_transport(self):
        self._check(self.lib.tdlb_debug_transport(self.h))


# ---------------------------------------------------------------------------
# Rushton-turbine geometry (host only), mirroring the calls main.cpp makes on
# RushtonTurbinePolarCPP (main.cpp:274-303, :409-426).
# ---------------------------------------------------------------------------
class Batch:
    """Many independent tanks on one GPU (``tdlb_batch_*``): one persistent
    fused launch steps every tank, then each tank's immersed-boundary pass;
    pairs of steps replay a captured CUDA graph.

    ``configs`` is a list of ``make_config`` keyword dicts (or Config
    structs), one per tank; all share one streaming scheme and one storage
    precision. ``tanks[t]`` is a ComputeUnit view of tank t for initialise,
    attach_rushton, set_markers and the read functions.
    """

    def __init__(self, configs, device: int = 0):
        self.lib = load_library()
        n = len(configs)
        arr = (Config * n)()
        for t, c in enumerate(configs):
            arr[t] = c if isinstance(c, Config) else make_config(**c)
        h = ctypes.c_void_p()
        rc = self.lib.tdlb_batch_create(arr, n, device, ctypes.byref(h))
        if rc != 0:
            raise TdlbError(rc, self.lib.tdlb_batch_last_error(None).decode())
        self.h = h
        self.tanks = []
        for t in range(n):
            th = ctypes.c_void_p()
            self._check(self.lib.tdlb_batch_tank(self.h, t, ctypes.byref(th)))
            self.tanks.append(ComputeUnit._borrowed(self.lib, th))

    def _check(self, rc: int):
        if rc != 0:
            raise TdlbError(rc, self.lib.tdlb_batch_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            for cu in self.tanks:
                cu.h = None
            self.lib.tdlb_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        return len(self.tanks)

    @property
    def ncell(self) -> int:
        return sum(cu.ncell for cu in self.tanks)

    def add(self, config) -> "ComputeUnit":
        """A new tank joins the batch (keyword dict or Config); returns its view."""
        cfg = config if isinstance(config, Config) else make_config(**config)
        idx = ctypes.c_int()
        self._check(self.lib.tdlb_batch_add(self.h, ctypes.byref(cfg), ctypes.byref(idx)))
        th = ctypes.c_void_p()
        self._check(self.lib.tdlb_batch_tank(self.h, idx.value, ctypes.byref(th)))
        cu = ComputeUnit._borrowed(self.lib, th)
        self.tanks.append(cu)
        return cu

    def adopt(self, cu: "ComputeUnit") -> "ComputeUnit":
        """A standalone ComputeUnit, already set up on its own stream, joins
        the batch as its last tank; the batch owns it from then on (closing
        `cu` no longer destroys it). Returns `cu`, now a view."""
        if not getattr(cu, "_owned", False) or not getattr(cu, "h", None):
            raise TdlbError(-5, "only a standalone, open ComputeUnit can be adopted")
        idx = ctypes.c_int()
        self._check(self.lib.tdlb_batch_adopt(self.h, cu.h, ctypes.byref(idx)))
        cu._owned = False
        self.tanks.append(cu)
        return cu

    def detach(self, index: int) -> "ComputeUnit":
        """Tank `index` leaves the batch without being destroyed; the returned
        ComputeUnit owns it again (closing it destroys the tank)."""
        th = ctypes.c_void_p()
        self._check(self.lib.tdlb_batch_detach(self.h, index, ctypes.byref(th)))
        cu = self.tanks.pop(index)
        cu.h = th
        cu._owned = True
        return cu

    def remove(self, index: int):
        """Tank `index` leaves the batch (its handle is destroyed)."""
        self._check(self.lib.tdlb_batch_remove(self.h, index))
        self.tanks.pop(index).h = None

    def set_shape(self, cells_per_thread: int, threads: int, blocks_per_sm: int):
        self._check(self.lib.tdlb_batch_set_shape(self.h, cells_per_thread, threads, blocks_per_sm))

    def shape(self):
        v, t, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.tdlb_batch_get_shape(self.h, ctypes.byref(v), ctypes.byref(t), ctypes.byref(b)))
        return v.value, t.value, b.value

    def autotune(self, trials: int = 3) -> float:
        ms = ctypes.c_double()
        self._check(self.lib.tdlb_batch_autotune(self.h, trials, ctypes.byref(ms)))
        return ms.value

    def run(self, steps: int, alpha: float, beta: float, graph: bool = True):
        fn = self.lib.tdlb_batch_run if graph else self.lib.tdlb_batch_run_eager
        self._check(fn(self.h, steps, alpha, beta))

    def synchronize(self):
        self._check(self.lib.tdlb_batch_synchronize(self.h))

    def kernel_launches(self) -> int:
        n = ctypes.c_longlong()
        self._check(self.lib.tdlb_batch_kernel_launches(self.h, ctypes.byref(n)))
        return n.value

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.lib.tdlb_batch_get_stream(self.h, ctypes.byref(s)))
        return s.value or 0


class Server:
    """The serving form (``tdlb_server_*``): submit tank solves from any
    thread; a native worker admits them by free HBM, keeps their lattices
    resident, batches them continuously and returns FP64 diagnostics (and,
    on request, the final density and velocity fields)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, max_active: int = 64, chunk_steps: int = 100):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.tdlb_server_create(device, hbm_budget, max_active, chunk_steps, ctypes.byref(h))
        if rc != 0:
            raise TdlbError(rc, self.lib.tdlb_server_last_error(None).decode())
        self.h = h
        self._fields = {}

    def _check(self, rc: int):
        if rc != 0:
            raise TdlbError(rc, self.lib.tdlb_server_last_error(self.h).decode())

    def submit(self, rid: int, edge, tip_speed: float, reynolds: float, steps: int, storage: str = "fp32",
               streaming: str = "Simple", les: bool = True, fields: bool = False):
        x, y, z = (edge, edge, edge) if isinstance(edge, int) else edge
        r = Request()
        r.id, r.x, r.y, r.z = rid, x, y, z
        r.tip_speed, r.reynolds, r.steps = tip_speed, reynolds, steps
        r.storage = {"fp32": STORAGE_FP32, "fp16": STORAGE_FP16, "bf16": STORAGE_BF16}[storage]
        r.streaming = STREAMING_SIMPLE if streaming == "Simple" else STREAMING_ESOTWIST
        r.les = int(les)
        if fields:
            out = {"rho": np.zeros((x, y, z), np.float32), "ux": np.zeros((x, y, z), np.float32),
                   "uy": np.zeros((x, y, z), np.float32), "uz": np.zeros((x, y, z), np.float32)}
            r.out_rho, r.out_ux, r.out_uy, r.out_uz = (out[k].ctypes.data for k in ("rho", "ux", "uy", "uz"))
            self._fields[rid] = out
        self._check(self.lib.tdlb_server_submit(self.h, ctypes.byref(r)))

    def poll(self, cap: int = 256):
        buf = (Result * cap)()
        n = ctypes.c_int()
        self._check(self.lib.tdlb_server_poll(self.h, buf, cap, ctypes.byref(n)))
        out = []
        for q in range(n.value):
            r = buf[q]
            d = {name: getattr(r, name) for name, _ in Result._fields_ if name != "pad"}
            d["momentum"], d["force"] = list(r.momentum), list(r.force)
            if r.id in self._fields:
                d["fields"] = self._fields.pop(r.id)
            out.append(d)
        return out

    def wait_idle(self, timeout_s: float = 3600.0):
        self._check(self.lib.tdlb_server_wait_idle(self.h, timeout_s))

    def stats(self) -> dict:
        st = ServerStats()
        self._check(self.lib.tdlb_server_get_stats(self.h, ctypes.byref(st)))
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "h", None):
            self.lib.tdlb_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


def lattice_bytes(x: int, y: int, z: int, storage: str = "fp32", streaming: str = "Simple") -> int:
    """Device bytes of a lattice (tdlb_lattice_bytes)."""
    lib = load_library()
    cfg = make_config(x=x, y=y, z=z, storage=storage, streaming=streaming)
    b = ctypes.c_int64()
    rc = lib.tdlb_lattice_bytes(ctypes.byref(cfg), ctypes.byref(b))
    if rc != 0:
        raise TdlbError(rc, "bad lattice size")
    return b.value


class RushtonTurbine:
    """Marker lists of the project's stirred-tank geometry for an x*y*z lattice."""

    def __init__(self, x: int, y: int, z: int, tip_speed: float = 0.1, startup_steps: int = 0, **spec):
        self.lib = load_library()
        self.spec = Rushton()
        self.spec.x, self.spec.y, self.spec.z = x, y, z
        self.spec.tip_speed = tip_speed
        self.spec.startup_steps = startup_steps
        for k, v in spec.items():
            setattr(self.spec, k, v)

    def _gen(self, fn, *args) -> np.ndarray:
        n = ctypes.c_size_t()
        rc = fn(ctypes.byref(self.spec), *args, None, 0, ctypes.byref(n))
        if rc:
            raise TdlbError(rc, "geometry query failed")
        out = np.zeros(n.value, MARKER_DTYPE)
        rc = fn(ctypes.byref(self.spec), *args, _p(out), n.value, ctypes.byref(n))
        if rc:
            raise TdlbError(rc, "geometry generation failed")
        return out

    def fixed(self) -> np.ndarray:
        return self._gen(self.lib.tdlb_rushton_fixed)

    def rotating_nonupdating(self, delta_angle: float) -> np.ndarray:
        return self._gen(self.lib.tdlb_rushton_rotating_nonupdating, ctypes.c_double(delta_angle))

    def rotating(self, angle: float, delta_angle: float) -> np.ndarray:
        return self._gen(self.lib.tdlb_rushton_rotating, ctypes.c_double(angle), ctypes.c_double(delta_angle))

    def increment(self, step: int) -> float:
        return self.lib.tdlb_rushton_impeller_increment(ctypes.byref(self.spec), step)

    def blade_outer_radius(self) -> int:
        return self.lib.tdlb_rushton_blade_outer_radius(ctypes.byref(self.spec))

    def forcing_list(self, angle: float, delta_angle: float, nonupdating_delta: float = None) -> np.ndarray:
        """fixed + rotating-non-updating + rotating, the order main.cpp:301-303 builds."""
        nd = delta_angle if nonupdating_delta is None else nonupdating_delta
        return np.concatenate([self.fixed(), self.rotating_nonupdating(nd), self.rotating(angle, delta_angle)])


def schedule_levels(markers, x: int, y: int, z: int):
    """Per-plane immersed-boundary level of each marker and the most levels in a plane."""
    lib = load_library()
    m = as_markers(markers)
    lev = np.zeros(len(m), np.int32)
    mx = ctypes.c_int32()
    rc = lib.tdlb_schedule_levels(_p(m), len(m), x, y, z, _p(lev), ctypes.byref(mx))
    if rc:
        raise TdlbError(rc, "schedule_levels failed")
    return lev, mx.value


def nu_from_reynolds(re: float, tip_speed: float, blade_outer_radius: int) -> float:
    """FlowParams::calcNuAndRe_m (FlowParams.hpp:65-70), in the reference's float arithmetic."""
    re_m = np.float32(float(np.float32(re)) * np.pi / 2.0)   # float * M_PI promotes to double
    return float(np.float32(np.float32(tip_speed) * np.float32(blade_outer_radius) / re_m))
