"""ctypes front end of the CPU checkers.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the snac_b200 package.

  Checker("port")       oracle/liboracle.so, the plain-C restatement
  Checker("reference")  oracle/_ref/libsnacref.so, the reference's own
                        hot-path sources compiled against oracle/refshim
  Checker("reference_mt", threads=n)
                        oracle/_ref/libsnacref_mt.so, the same sources with
                        the driver's element and node loops on n threads
                        (bitwise equal to "reference"): the all-cores CPU
                        baseline
Both take the product's descriptor (snac_b200.abi.SnacConfig) and expose the
same calls, so a test can run the GPU path and either checker side by side.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

from snac_b200.abi import NT, Desc, Scalars, SnacConfig, State, StateView

HERE = os.path.dirname(os.path.abspath(__file__))
PATHS = {"port": os.path.join(HERE, "liboracle.so"),
         "reference": os.path.join(HERE, "_ref", "libsnacref.so"),
         "reference_mt": os.path.join(HERE, "_ref", "libsnacref_mt.so"),
         "plugin_host": os.path.join(HERE, "_ref", "libsnaccuda_host.so")}
PREFIX = {"port": "so_", "reference": "ref_", "reference_mt": "ref_", "plugin_host": "ref_"}


def snac_tree() -> str:
    """The SNAC source tree the reference checkers compile from: $SNAC_REF when
    set, else reference/Snac beside this repository's directory."""
    env = os.environ.get("SNAC_REF")
    if env:
        return env
    return os.path.normpath(os.path.join(HERE, "..", "..", "reference", "Snac"))


def build(kind: str = "port") -> str:
    """Compile the checker with oracle/Makefile if it is missing."""
    path = PATHS[kind]
    if not os.path.exists(path):
        target = {"port": "all", "plugin_host": "plugin"}.get(kind, "ref")
        subprocess.run(["make", "-s", "-C", HERE, target, f"SNAC_REF={snac_tree()}"], check=True)
    return path


def available(kind: str) -> bool:
    return os.path.exists(PATHS[kind])


_LIBS = {}


def _lib(kind: str):
    if kind not in _LIBS:
        lib = C.CDLL(build(kind))
        p = PREFIX[kind]
        vp = C.c_void_p
        lib_fn = lambda n: getattr(lib, p + n)  # noqa: E731
        lib_fn("create").restype = vp
        lib_fn("create").argtypes = [C.POINTER(Desc), C.POINTER(C.c_int)]
        lib_fn("destroy").argtypes = [vp]
        for n in ("time_step_zero", "begin_step", "loop_elements_energy", "loop_nodes_energy",
                  "calc_stresses", "loop_nodes_momentum", "loop_elements_momentum", "sync"):
            lib_fn(n).argtypes = [vp]
            lib_fn(n).restype = C.c_int
        if kind == "port":
            lib_fn("node_forces").argtypes = [vp]
            lib_fn("node_forces").restype = C.c_int
        else:
            lib_fn("set_threads").argtypes = [C.c_int]
            lib_fn("threads").restype = C.c_int
            if kind in ("reference", "reference_mt"):
                lib_fn("set_verbatim_bc").argtypes = [vp, C.c_int]
        lib_fn("step").argtypes = [vp, C.c_int]
        lib_fn("step").restype = C.c_int
        lib_fn("get_state").argtypes = [vp, C.POINTER(StateView)]
        lib_fn("set_state").argtypes = [vp, C.POINTER(StateView)]
        lib_fn("scalars").argtypes = [vp, C.POINTER(Scalars)]
        lib_fn("set_dt").argtypes = [vp, C.c_double]
        lib_fn("last_error").argtypes = [vp]
        lib_fn("last_error").restype = C.c_char_p
        dp = C.POINTER(C.c_double)
        lib_fn("get_geometry").argtypes = [vp, dp, dp, dp]
        lib_fn("get_element_scalars").argtypes = [vp, dp, dp, dp, dp, dp, dp]
        lib_fn("get_tet_fields").argtypes = [vp, dp, dp, dp, dp]
        lib_fn("get_node_fields").argtypes = [vp, dp, dp]
        _LIBS[kind] = lib
    return _LIBS[kind]


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


class Checker:
    """One CPU model run (a Snac_Context)."""

    def __init__(self, cfg: SnacConfig, kind: str = "port", threads: int = 1):
        self.kind = kind
        self.cfg = cfg
        self.lib = _lib(kind)
        self._f = lambda n: getattr(self.lib, PREFIX[kind] + n)  # noqa: E731
        if kind != "port":
            self._f("set_threads")(int(threads))
        self.threads = self._f("threads")() if kind != "port" else 1
        self._desc = cfg.desc()
        st = C.c_int(0)
        self.h = self._f("create")(C.byref(self._desc), C.byref(st))
        self.status = st.value
        if not self.h:
            raise RuntimeError(f"{kind} checker: create failed with status {st.value}")
        self.ne, self.nn = cfg.n_elements, cfg.n_nodes

    def close(self):
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, name, *args) -> int:
        return self._f(name)(self.h, *args)

    def time_step_zero(self) -> int:
        return self._call("time_step_zero")

    def step(self, n: int = 1) -> int:
        return self._call("step", int(n))

    def begin_step(self):
        return self._call("begin_step")

    def loop_elements_energy(self):
        return self._call("loop_elements_energy")

    def loop_nodes_energy(self):
        return self._call("loop_nodes_energy")

    def calc_stresses(self):
        return self._call("calc_stresses")

    def loop_nodes_momentum(self):
        return self._call("loop_nodes_momentum")

    def loop_elements_momentum(self):
        return self._call("loop_elements_momentum")

    def sync(self):
        return self._call("sync")

    def node_forces(self):
        """Snac_Force for every node, without the node update (port only)."""
        return self._call("node_forces")

    def set_dt(self, dt: float):
        self._f("set_dt")(self.h, C.c_double(dt))

    def set_verbatim_bc(self, on: bool = True):
        """Compiled reference only: the boundary conditions' ApplyToIndex
        searches its index table linearly, as StGermain's does
        (VariableCondition.c:449-463), instead of the O(1) per-node mask
        (same results, the reference's cost)."""
        if self.kind not in ("reference", "reference_mt"):
            raise ValueError("the verbatim search is an option of the compiled reference")
        self._f("set_verbatim_bc")(self.h, 1 if on else 0)

    def last_error(self) -> str:
        return self._f("last_error")(self.h).decode()

    def state(self) -> State:
        s = State.empty(self.ne, self.nn)
        v = s.view()
        self._f("get_state")(self.h, C.byref(v))
        return s

    def set_state(self, s: State, fields=None):
        v = s.view(fields)
        self._f("set_state")(self.h, C.byref(v))

    def scalars(self) -> Scalars:
        o = Scalars()
        self._f("scalars")(self.h, C.byref(o))
        return o

    def geometry(self):
        vol = np.zeros((self.ne, NT))
        area = np.zeros((self.ne, NT, 4))
        nrm = np.zeros((self.ne, NT, 4, 3))
        self._f("get_geometry")(self.h, _p(vol), _p(area), _p(nrm))
        return vol, area, nrm

    def element_scalars(self):
        out = [np.zeros(self.ne) for _ in range(6)]
        self._f("get_element_scalars")(self.h, *[_p(a) for a in out])
        return dict(zip(("volume", "strain_rate", "stress", "hydro_pressure", "aps", "min_length_scale"), out))

    def tet_fields(self):
        sr = np.zeros((self.ne, NT, 6))
        sn = np.zeros((self.ne, NT, 6))
        den = np.zeros((self.ne, NT))
        at = np.zeros((self.ne, NT))
        self._f("get_tet_fields")(self.h, _p(sr), _p(sn), _p(den), _p(at))
        return {"strain_rate": sr, "strain": sn, "density": den, "avg_temp": at}

    def node_fields(self):
        mass = np.zeros(self.nn)
        bal = np.zeros((self.nn, 3))
        self._f("get_node_fields")(self.h, _p(mass), _p(bal))
        return {"mass": mass, "balance": bal}


class PluginHost(Checker):
    """A Snac_Context of the reference sources (as Checker("reference")) into
    which the SnacCuda plugin (snac_b200/plugin) is loaded the way
    StGermain's PluginLoader loads it, then driven the way AbstractContext
    drives a context: Initialise, steps of Dt / Solve / Sync, Dump, each
    through whatever hooks the entry points hold.  Test infrastructure for
    the plugin; stepping needs a GPU (the plugin's hooks call libsnac_b200)."""

    def __init__(self, cfg: SnacConfig):
        super().__init__(cfg, "plugin_host")
        f = self._f
        vp = C.c_void_p
        for n in ("host_load_plugin",):
            f(n).argtypes = [vp, C.c_char_p]
            f(n).restype = C.c_int
        for n in ("host_initialise", "host_dump"):
            f(n).argtypes = [vp]
            f(n).restype = C.c_int
        f("host_step").argtypes = [vp, C.c_int]
        f("host_step").restype = C.c_int
        f("host_hooks").argtypes = [vp, C.c_char_p, C.c_char_p, C.c_int]
        f("host_hooks").restype = C.c_int
        f("host_context").argtypes = [vp]
        f("host_context").restype = vp
        f("host_extension").argtypes = [vp, C.c_char_p]
        f("host_extension").restype = vp

    def load_plugin(self, name: str = "SnacCuda") -> int:
        return self._f("host_load_plugin")(self.h, name.encode())

    def initialise(self) -> int:
        return self._f("host_initialise")(self.h)

    def host_step(self, n: int = 1) -> int:
        return self._f("host_step")(self.h, int(n))

    def dump(self) -> int:
        return self._f("host_dump")(self.h)

    def hooks(self, entry_point: str):
        buf = C.create_string_buffer(1024)
        self._f("host_hooks")(self.h, entry_point.encode(), buf, 1024)
        return buf.value.decode().split(",") if buf.value else []

    def context_ptr(self) -> int:
        return self._f("host_context")(self.h)

    def extension_ptr(self, name: str) -> int:
        return self._f("host_extension")(self.h, name.encode())
