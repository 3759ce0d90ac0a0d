"""Python front end of the CUDA library (libsnac_b200.so) through its C ABI.

SnacContext mirrors the reference's Snac_Context life cycle
(Snac/libSnac/src/Context.c): construction applies the initial conditions,
time_step_zero() is Snac_Context_TimeStepZero, step(n) runs n
_AbstractContext_Step's (Solve + Sync), and the loop-level methods are the
entry points a StGermain plugin replaces.  Every call goes to the CUDA
library; there is no CPU path here.  If the library is missing or no GPU is
visible, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

from .abi import NT, STATUS_NAMES, BatchTuning, Desc, KernelTime, Scalars, SnacConfig, State, StateView

HERE = os.path.dirname(os.path.abspath(__file__))
# $SNAC_B200_LIB selects another build of the library (e.g. a variant built
# with different compile-time options, for comparison)
LIB_PATH = os.environ.get("SNAC_B200_LIB") or os.path.join(HERE, "libsnac_b200.so")


class SnacError(RuntimeError):
    def __init__(self, code: int, msg: str, index: int = -1):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code
        self.index = index


_LIB = None


def load_library(path: str = LIB_PATH):
    """Load libsnac_b200.so (raises OSError if it was not built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: run __graft_entry__.build() (or python -m snac_b200.build)")
    lib = C.CDLL(path)
    vp = C.c_void_p
    lib.snac_gpu_create.argtypes = [C.POINTER(Desc), C.POINTER(vp)]
    lib.snac_gpu_create.restype = C.c_int
    lib.snac_gpu_destroy.argtypes = [vp]
    lib.snac_gpu_destroy.restype = None
    for n in ("time_step_zero", "begin_step", "loop_elements_energy", "loop_nodes_energy", "calc_stresses",
              "loop_nodes_momentum", "loop_elements_momentum", "sync"):
        f = getattr(lib, "snac_gpu_" + n)
        f.argtypes = [vp]
        f.restype = C.c_int
    lib.snac_gpu_step.argtypes = [vp, C.c_int]
    lib.snac_gpu_step.restype = C.c_int
    lib.snac_gpu_time_steps.argtypes = [vp, C.c_int, vp, C.c_size_t, C.POINTER(C.c_double)]
    lib.snac_gpu_time_steps.restype = C.c_int
    lib.snac_gpu_upload.argtypes = [vp, C.POINTER(StateView)]
    lib.snac_gpu_upload.restype = C.c_int
    lib.snac_gpu_download.argtypes = [vp, C.POINTER(StateView)]
    lib.snac_gpu_download.restype = C.c_int
    lib.snac_gpu_step_host.argtypes = [vp, C.POINTER(StateView), C.POINTER(StateView), C.c_int]
    lib.snac_gpu_step_host.restype = C.c_int
    lib.snac_gpu_scalars.argtypes = [vp, C.POINTER(Scalars)]
    lib.snac_gpu_scalars.restype = C.c_int
    lib.snac_gpu_set_dt.argtypes = [vp, C.c_double]
    lib.snac_gpu_set_dt.restype = C.c_int
    lib.snac_gpu_last_error.argtypes = [vp]
    lib.snac_gpu_last_error.restype = C.c_char_p
    lib.snac_gpu_error_index.argtypes = [vp]
    lib.snac_gpu_error_index.restype = C.c_longlong
    lib.snac_gpu_sizes.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    lib.snac_gpu_sizes.restype = C.c_int
    lib.snac_gpu_launch_count.argtypes = [vp]
    lib.snac_gpu_launch_count.restype = C.c_longlong
    lib.snac_gpu_stream.argtypes = [vp]
    lib.snac_gpu_stream.restype = vp
    lib.snac_gpu_profile_step.argtypes = [vp, C.POINTER(KernelTime), C.c_int]
    lib.snac_gpu_profile_step.restype = C.c_int
    lib.snac_gpu_selftest_division.argtypes = [C.c_longlong, C.c_ulonglong, C.POINTER(C.c_longlong)]
    lib.snac_gpu_selftest_division.restype = C.c_int
    lib.snac_gpu_device_count.argtypes = []
    lib.snac_gpu_device_count.restype = C.c_int
    lib.snac_gpu_output_open.argtypes = [vp, C.c_char_p, C.c_uint, C.c_uint, C.c_uint, C.c_uint]
    lib.snac_gpu_output_open.restype = C.c_int
    lib.snac_gpu_write_output.argtypes = [vp]
    lib.snac_gpu_write_output.restype = C.c_int
    lib.snac_gpu_output_close.argtypes = [vp]
    lib.snac_gpu_output_close.restype = C.c_int
    # batched ensembles
    lib.snac_gpu_batch_create.argtypes = [C.POINTER(Desc), C.c_int, C.POINTER(vp)]
    lib.snac_gpu_batch_create.restype = C.c_int
    lib.snac_gpu_batch_destroy.argtypes = [vp]
    lib.snac_gpu_batch_destroy.restype = None
    lib.snac_gpu_batch_time_step_zero.argtypes = [vp]
    lib.snac_gpu_batch_time_step_zero.restype = C.c_int
    for n in ("step", "step_each"):
        f = getattr(lib, "snac_gpu_batch_" + n)
        f.argtypes = [vp, C.c_int]
        f.restype = C.c_int
    lib.snac_gpu_batch_model.argtypes = [vp, C.c_int]
    lib.snac_gpu_batch_model.restype = vp
    lib.snac_gpu_batch_size.argtypes = [vp]
    lib.snac_gpu_batch_size.restype = C.c_int
    lib.snac_gpu_batch_get_tuning.argtypes = [vp, C.POINTER(BatchTuning)]
    lib.snac_gpu_batch_get_tuning.restype = C.c_int
    lib.snac_gpu_batch_set_tuning.argtypes = [vp, C.POINTER(BatchTuning)]
    lib.snac_gpu_batch_set_tuning.restype = C.c_int
    lib.snac_gpu_batch_time_steps.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_double)]
    lib.snac_gpu_batch_time_steps.restype = C.c_int
    lib.snac_gpu_batch_last_error.argtypes = [vp]
    lib.snac_gpu_batch_last_error.restype = C.c_char_p
    lib.snac_gpu_batch_error_model.argtypes = [vp]
    lib.snac_gpu_batch_error_model.restype = C.c_int
    lib.snac_gpu_batch_launch_count.argtypes = [vp]
    lib.snac_gpu_batch_launch_count.restype = C.c_longlong
    lib.snac_gpu_batch_stream.argtypes = [vp]
    lib.snac_gpu_batch_stream.restype = vp
    _LIB = lib
    return lib


class SnacContext:
    """One model on the GPU (one snac_gpu handle)."""

    owned = True

    @classmethod
    def borrowed(cls, cfg: SnacConfig, handle: int, owner) -> "SnacContext":
        """A view of a model whose handle belongs to `owner` (a batch): same
        methods, but closing it does not destroy the model."""
        self = cls.__new__(cls)
        self.lib = load_library()
        self.cfg = cfg
        self.h = C.c_void_p(handle)
        self.ne, self.nn = cfg.n_elements, cfg.n_nodes
        self.owned = False
        self._owner = owner
        return self

    def __init__(self, cfg: SnacConfig):
        self.lib = load_library()
        self.cfg = cfg
        self._desc = cfg.desc()
        self.h = C.c_void_p()
        rc = self.lib.snac_gpu_create(C.byref(self._desc), C.byref(self.h))
        if rc != 0:
            msg = self.lib.snac_gpu_last_error(self.h).decode() if self.h else ""
            if self.h:
                self.lib.snac_gpu_destroy(self.h)
                self.h = C.c_void_p()
            raise SnacError(rc, msg or "snac_gpu_create failed")
        self.ne, self.nn = cfg.n_elements, cfg.n_nodes

    # -- lifetime ---------------------------------------------------------------------
    def close(self):
        if self.h:
            if self.owned:
                self.lib.snac_gpu_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int) -> int:
        if rc != 0:
            raise SnacError(rc, self.lib.snac_gpu_last_error(self.h).decode(), self.lib.snac_gpu_error_index(self.h))
        return rc

    # -- the reference's step structure ------------------------------------------------
    def time_step_zero(self):
        return self._check(self.lib.snac_gpu_time_step_zero(self.h))

    def step(self, n: int = 1):
        return self._check(self.lib.snac_gpu_step(self.h, int(n)))

    def time_steps(self, n: int, flush_ptr: int = 0, flush_bytes: int = 0):
        """n steps, each after a write of flush_bytes at flush_ptr (an L2
        flush) and timed alone with CUDA events: [ms of step i]."""
        ms = (C.c_double * int(n))()
        self._check(self.lib.snac_gpu_time_steps(self.h, int(n), C.c_void_p(flush_ptr or None), int(flush_bytes), ms))
        return list(ms)

    def begin_step(self):
        return self._check(self.lib.snac_gpu_begin_step(self.h))

    def loop_elements_energy(self):
        return self._check(self.lib.snac_gpu_loop_elements_energy(self.h))

    def loop_nodes_energy(self):
        return self._check(self.lib.snac_gpu_loop_nodes_energy(self.h))

    def calc_stresses(self):
        return self._check(self.lib.snac_gpu_calc_stresses(self.h))

    def loop_nodes_momentum(self):
        return self._check(self.lib.snac_gpu_loop_nodes_momentum(self.h))

    def loop_elements_momentum(self):
        return self._check(self.lib.snac_gpu_loop_elements_momentum(self.h))

    def sync(self):
        return self._check(self.lib.snac_gpu_sync(self.h))

    def solve(self):
        """_Snac_Context_Solve + Sync for one step, hook by hook."""
        self.begin_step()
        self.loop_elements_energy()
        self.loop_nodes_energy()
        self.calc_stresses()
        self.loop_nodes_momentum()
        self.loop_elements_momentum()
        self.sync()

    # -- state --------------------------------------------------------------------------
    @property
    def keeps_plastic_strain_tensor(self) -> bool:
        """The visco-plastic hook with a Drucker-Prager phase keeps a per-tet
        plastic strain tensor; other models have none (it reads as zero)."""
        return self.cfg.plugin == "SnacViscoPlastic" and any(
            m.get("yieldcriterion", "mohrcoulomb") != "mohrcoulomb" for m in self.cfg.materials)

    def state(self, out: Optional[State] = None) -> State:
        """The state at the end of the last step (into `out` if given, e.g. pinned buffers)."""
        s = out if out is not None else State.empty(self.ne, self.nn)
        v = s.view()
        if not self.keeps_plastic_strain_tensor:
            v.plastic_strain_tensor = None  # nothing to copy: the State's tensor stays as it is (zero)
        self._check(self.lib.snac_gpu_download(self.h, C.byref(v)))
        return s

    def set_state(self, s: State, fields: Optional[list] = None):
        v = s.view(fields)
        self._check(self.lib.snac_gpu_upload(self.h, C.byref(v)))

    def step_host(self, s_in: State, s_out: State, fields_in: Optional[list] = None,
                  fields_out: Optional[list] = None, chunks: int = 0) -> State:
        """One step of a host-held state: upload `fields_in` of s_in, one step,
        download `fields_out` into s_out (same bits as set_state + step(1) +
        state), with the transfers overlapped slab by slab (snac_gpu_step_host).
        Without an explicit list, the step's state moves: coordinates,
        velocities, stresses, the hooks' per-tet state and the temperature."""
        default = ["coord", "velocity", "stress", "plastic_strain", "viscosity"]
        if self.cfg.temperature:
            default.append("temperature")
        if self.keeps_plastic_strain_tensor:
            default.append("plastic_strain_tensor")
        vi = s_in.view(fields_in if fields_in is not None else default)
        vo = s_out.view(fields_out if fields_out is not None else default)
        self._check(self.lib.snac_gpu_step_host(self.h, C.byref(vi), C.byref(vo), int(chunks)))
        return s_out

    def scalars(self) -> Scalars:
        o = Scalars()
        self._check(self.lib.snac_gpu_scalars(self.h, C.byref(o)))
        return o

    def set_dt(self, dt: float):
        self._check(self.lib.snac_gpu_set_dt(self.h, C.c_double(dt)))

    # -- output files in the reference's format ---------------------------------------
    def output_open(self, path: str, rank: int = 0, dump_every: int = 1, checkpoint_every: int = 0,
                    max_time_steps: int = 0):
        """Context.c _Snac_Context_InitDump / InitCheckpoint: open the dump files."""
        return self._check(self.lib.snac_gpu_output_open(self.h, path.encode(), rank, dump_every,
                                                          checkpoint_every, max_time_steps))

    def write_output(self):
        """_Snac_Context_WriteOutput for the current timeStep (asynchronous file writes)."""
        return self._check(self.lib.snac_gpu_write_output(self.h))

    def output_close(self):
        return self._check(self.lib.snac_gpu_output_close(self.h))

    def profile_step(self):
        """One step kernel by kernel with CUDA events: [(kernel name, ms)]."""
        buf = (KernelTime * 32)()
        n = self.lib.snac_gpu_profile_step(self.h, buf, 32)
        if n < 0:
            self._check(n)
        return [(buf[i].name.decode(), buf[i].ms) for i in range(n)]

    @property
    def launches(self) -> int:
        return int(self.lib.snac_gpu_launch_count(self.h))

    @property
    def stream(self) -> int:
        return int(self.lib.snac_gpu_stream(self.h) or 0)
