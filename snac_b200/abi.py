"""ctypes mirror of include/snac_gpu.h (structs, constants) plus helpers that
build a descriptor from the reference's own dictionary keys.

The key names follow the StGermain/SNAC input dictionary read by
Snac/libSnac/src/Context.c:345-391 (dtType, timeStep), :752-761
(strain_inert, topo_kappa), :816-819 (gravity, demf) and :826-914 (the
per-phase keys density, alpha, beta, lambda, mu, nsegments, plstrain<i>,
frictionAngle<i>, dilationAngle<i>, cohesion<i>, ten_off, vis_min, vis_max,
refvisc, refsrate, reftemp, activationE, srexponent, thermal_conduct,
heatCapacity).  Unlike the reference, no float-literal default is applied:
every key a workload needs must be given (the reference's defaults are
available as REFERENCE_DEFAULTS, float-rounded the way the reference reads
them).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional, Sequence

import numpy as np

ABI_VERSION = 2

OK = 0
EINVAL = -1
ENOMEM = -2
ECUDA = -3
ENAN = -4
EVOLUME = -5
EMATERIAL = -6
EPHYSICS = -7
ETIMEDOUT = -8
ENOTSUP = -9
ESTATE = -10
ENODEV = -11
STATUS_NAMES = {0: "OK", -1: "EINVAL", -2: "ENOMEM", -3: "ECUDA", -4: "ENAN", -5: "EVOLUME",
                -6: "EMATERIAL", -7: "EPHYSICS", -8: "ETIMEDOUT", -9: "ENOTSUP", -10: "ESTATE",
                -11: "ENODEV"}

DT_CONSTANT, DT_DYNAMIC, DT_WAVE = 0, 1, 2
DT_TYPES = {"constant": DT_CONSTANT, "dynamic": DT_DYNAMIC, "wave": DT_WAVE}

ELASTIC, PLASTIC, MAXWELL, VISCOPLASTIC = 0x1, 0x2, 0x4, 0x8
PLUGINS = {"SnacElastic": ELASTIC, "SnacPlastic": PLASTIC, "SnacMaxwell": MAXWELL,
           "SnacViscoPlastic": VISCOPLASTIC}

WALL_BACK, WALL_LEFT, WALL_BOTTOM, WALL_RIGHT, WALL_TOP, WALL_FRONT, WALL_ALL = range(7)
WALLS = {"back": WALL_BACK, "left": WALL_LEFT, "bottom": WALL_BOTTOM, "right": WALL_RIGHT,
         "top": WALL_TOP, "front": WALL_FRONT, "all": WALL_ALL}

MAX_SEGMENTS = 8
NT = 10  # tetrahedra per hex

F32 = lambda x: float(np.float32(x))  # noqa: E731  value of a C float literal promoted to double

# Context.c:345-914 defaults as the reference reads them (float literals rounded)
REFERENCE_DEFAULTS: Dict[str, Any] = {
    "strain_inert": F32(1.0e-5), "gravity": F32(9.81), "demf": F32(0.8), "topo_kappa": F32(5.0e-06),
    "density": 2700.0, "alpha": F32(3.0e-05), "beta": 0.0, "lambda": F32(3.0e+10), "mu": F32(3.0e+10),
    "nsegments": 2, "ten_off": 0.0, "vis_min": 1.0e18, "vis_max": 3.0e27, "refvisc": 1.0e19,
    "refsrate": 1.0e-15, "reftemp": 1400.0, "activationE": 5.4e03, "srexponent": 1.0,
    "thermal_conduct": 2.0, "heatCapacity": 1000.0,
}


class Material(C.Structure):
    _fields_ = [
        ("density", C.c_double), ("alpha", C.c_double), ("beta", C.c_double),
        ("lambda_", C.c_double), ("mu", C.c_double),
        ("nsegments", C.c_int), ("yield_mohr_coulomb", C.c_int),
        ("plstrain", C.c_double * (MAX_SEGMENTS + 1)),
        ("friction_angle", C.c_double * (MAX_SEGMENTS + 1)),
        ("dilation_angle", C.c_double * (MAX_SEGMENTS + 1)),
        ("cohesion", C.c_double * (MAX_SEGMENTS + 1)),
        ("ten_off", C.c_double),
        ("vis_min", C.c_double), ("vis_max", C.c_double), ("refvisc", C.c_double),
        ("refsrate", C.c_double), ("reftemp", C.c_double),
        ("activation_e", C.c_double), ("srexponent", C.c_double),
        ("thermal_conduct", C.c_double), ("heat_capacity", C.c_double),
    ]


class WallBC(C.Structure):
    _fields_ = [("wall", C.c_int), ("mask", C.c_int), ("value", C.c_double * 3)]


_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)


class Desc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("min", C.c_double * 3), ("max", C.c_double * 3),
        ("node_coords", _DP),
        ("dt_type", C.c_int), ("dt", C.c_double), ("strain_inert", C.c_double),
        ("gravity", C.c_double), ("demf", C.c_double),
        ("constitutive", C.c_int), ("temperature", C.c_int), ("compute_thermal_stress", C.c_int),
        ("hydrostatic_ic", C.c_int), ("temperature_sweep_ic", C.c_int),
        ("top_temp", C.c_double), ("bottom_temp", C.c_double),
        ("n_materials", C.c_int), ("materials", C.POINTER(Material)),
        ("element_material", _IP),
        ("element_cohesion_scale", _DP), ("element_friction_scale", _DP), ("element_visc_scale", _DP),
        ("n_velocity_bcs", C.c_int), ("velocity_bcs", C.POINTER(WallBC)),
        ("n_temperature_bcs", C.c_int), ("temperature_bcs", C.POINTER(WallBC)),
        ("init_velocity", _DP), ("init_temperature", _DP), ("init_stress", _DP),
        ("winkler", C.c_int), ("traction_bc", C.c_int),
        ("topo_kappa", C.c_double), ("topo_grad_criterion", C.c_double),
        ("pisos", C.c_double), ("rzbo", C.c_double),
        ("node_velocity_bc_mask", C.POINTER(C.c_ubyte)), ("node_velocity_bc_value", _DP),
        ("node_temperature_bc_mask", C.POINTER(C.c_ubyte)), ("node_temperature_bc_value", _DP),
        ("dp_max_iterations", _IP), ("dp_tolerance", _DP),
    ]


class StateView(C.Structure):
    _fields_ = [("coord", _DP), ("velocity", _DP), ("stress", _DP), ("plastic_strain", _DP),
                ("viscosity", _DP), ("temperature", _DP), ("force", _DP), ("inertial_mass", _DP),
                ("plastic_strain_tensor", _DP)]


class KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 40), ("ms", C.c_double)]


class BatchTuning(C.Structure):
    _fields_ = [("node_threads", C.c_int), ("minls_threads", C.c_int), ("elem_blocks_per_sm", C.c_int),
                ("node_blocks_per_sm", C.c_int), ("steps_per_graph", C.c_int), ("order", C.c_int),
                ("split_classes", C.c_int)]

    def as_dict(self) -> Dict[str, int]:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}

    @classmethod
    def from_dict(cls, d: Dict[str, int]) -> "BatchTuning":
        t = cls()
        for k, _ in cls._fields_:
            setattr(t, k, int(d[k]))
        return t


class Scalars(C.Structure):
    _fields_ = [("dt", C.c_double), ("min_length_scale", C.c_double), ("vmax", C.c_double),
                ("speed_of_sound", C.c_double), ("time_step", C.c_longlong), ("current_time", C.c_double)]


def _dptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_DP)


def material_from_dict(d: Dict[str, Any]) -> Material:
    """One phase from reference keys (Context.c:826-914)."""
    m = Material()
    m.density = float(d["density"])
    m.alpha = float(d.get("alpha", 0.0))
    m.beta = float(d.get("beta", 0.0))
    m.lambda_ = float(d["lambda"])
    m.mu = float(d["mu"])
    nseg = int(d.get("nsegments", 1))
    if nseg > MAX_SEGMENTS:
        raise ValueError(f"nsegments={nseg} > {MAX_SEGMENTS}")
    m.nsegments = nseg
    m.yield_mohr_coulomb = 1 if d.get("yieldcriterion", "mohrcoulomb") == "mohrcoulomb" else 0
    for i in range(nseg + 1):
        m.plstrain[i] = float(d.get(f"plstrain{i}", 0.0))
        m.friction_angle[i] = float(d.get(f"frictionAngle{i}", 0.0))
        m.dilation_angle[i] = float(d.get(f"dilationAngle{i}", 0.0))
        m.cohesion[i] = float(d.get(f"cohesion{i}", 0.0))
    m.ten_off = float(d.get("ten_off", 0.0))
    m.vis_min = float(d.get("vis_min", REFERENCE_DEFAULTS["vis_min"]))
    m.vis_max = float(d.get("vis_max", REFERENCE_DEFAULTS["vis_max"]))
    m.refvisc = float(d.get("refvisc", REFERENCE_DEFAULTS["refvisc"]))
    m.refsrate = float(d.get("refsrate", REFERENCE_DEFAULTS["refsrate"]))
    m.reftemp = float(d.get("reftemp", REFERENCE_DEFAULTS["reftemp"]))
    m.activation_e = float(d.get("activationE", REFERENCE_DEFAULTS["activationE"]))
    m.srexponent = float(d.get("srexponent", REFERENCE_DEFAULTS["srexponent"]))
    m.thermal_conduct = float(d.get("thermal_conduct", REFERENCE_DEFAULTS["thermal_conduct"]))
    m.heat_capacity = float(d.get("heatCapacity", REFERENCE_DEFAULTS["heatCapacity"]))
    return m


@dataclass
class SnacConfig:
    """A SNAC run in the reference's vocabulary; holds the numpy buffers the
    descriptor points into, so keep it alive while a handle uses it."""

    nx: int
    ny: int
    nz: int
    min: Sequence[float]
    max: Sequence[float]
    dtType: str = "dynamic"
    timeStep: float = 0.0
    strain_inert: float = 1.0e-5
    gravity: float = 0.0
    demf: float = 0.8
    plugin: str = "SnacElastic"           # the one constitutive plugin
    temperature: bool = False             # SnacTemperature loaded
    computeThermalStress: bool = False
    hydrostatic_ic: bool = False          # SnacHydroStaticIC loaded
    winkler: bool = False                 # SnacWinklerForce loaded (bottom support)
    traction_bc: bool = False             # SnacTractionBC loaded (right-wall stress)
    topo_kappa: float = 0.0               # surface-topography diffusivity (0 = off)
    topoGradCriterion: float = 1.0e-16
    materials: List[Dict[str, Any]] = field(default_factory=list)
    element_material: Optional[np.ndarray] = None
    element_cohesion_scale: Optional[np.ndarray] = None
    element_friction_scale: Optional[np.ndarray] = None
    element_visc_scale: Optional[np.ndarray] = None
    velocityBCs: List[Dict[str, Any]] = field(default_factory=list)   # {"wall":..,"vx":..,...}
    temperatureBCs: List[Dict[str, Any]] = field(default_factory=list)  # {"wall":..,"T":..}
    init_velocity: Optional[np.ndarray] = None
    init_temperature: Optional[np.ndarray] = None
    temperature_sweep: Optional[Sequence[float]] = None  # (topTemp, bottomTemp)
    init_stress: Optional[np.ndarray] = None
    node_coords: Optional[np.ndarray] = None
    _keep: List[Any] = field(default_factory=list, repr=False)

    @property
    def n_elements(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def n_nodes(self) -> int:
        return (self.nx + 1) * (self.ny + 1) * (self.nz + 1)

    def desc(self) -> Desc:
        d = Desc()
        keep: List[Any] = []
        d.abi_version = ABI_VERSION
        d.nx, d.ny, d.nz = self.nx, self.ny, self.nz
        for q in range(3):
            d.min[q] = float(self.min[q])
            d.max[q] = float(self.max[q])
        d.dt_type = DT_TYPES[self.dtType]
        d.dt = float(self.timeStep)
        d.strain_inert = float(self.strain_inert)
        d.gravity = float(self.gravity)
        d.demf = float(self.demf)
        d.constitutive = PLUGINS[self.plugin]
        d.temperature = int(bool(self.temperature))
        d.compute_thermal_stress = int(bool(self.computeThermalStress))
        d.hydrostatic_ic = int(bool(self.hydrostatic_ic))
        d.winkler = int(bool(self.winkler))
        d.traction_bc = int(bool(self.traction_bc))
        d.topo_kappa = float(self.topo_kappa)
        d.topo_grad_criterion = float(self.topoGradCriterion)
        if self.temperature_sweep is not None:
            d.temperature_sweep_ic = 1
            d.top_temp, d.bottom_temp = (float(x) for x in self.temperature_sweep)
        mats = (Material * len(self.materials))(*[material_from_dict(m) for m in self.materials])
        keep.append(mats)
        d.n_materials = len(self.materials)
        d.materials = mats

        def arr(a, dtype, n=None):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dtype)
            if n is not None and a.size != n:
                raise ValueError(f"array of size {a.size}, expected {n}")
            keep.append(a)
            return a.ctypes.data_as(_IP if dtype == np.int32 else _DP)

        ne, nn = self.n_elements, self.n_nodes
        if any(m.get("yieldcriterion", "mohrcoulomb") != "mohrcoulomb" for m in self.materials):
            d.dp_max_iterations = arr([int(m.get("maxiterations", 1)) for m in self.materials], np.int32)
            d.dp_tolerance = arr([float(m.get("constitutivetolerance", 1.0e-3)) for m in self.materials], np.float64)
        d.element_material = arr(self.element_material, np.int32, ne)
        d.element_cohesion_scale = arr(self.element_cohesion_scale, np.float64, ne)
        d.element_friction_scale = arr(self.element_friction_scale, np.float64, ne)
        d.element_visc_scale = arr(self.element_visc_scale, np.float64, ne)
        d.node_coords = arr(self.node_coords, np.float64, nn * 3)
        d.init_velocity = arr(self.init_velocity, np.float64, nn * 3)
        d.init_temperature = arr(self.init_temperature, np.float64, nn)
        d.init_stress = arr(self.init_stress, np.float64, ne * NT * 6)
        vb = (WallBC * max(1, len(self.velocityBCs)))()
        for i, bc in enumerate(self.velocityBCs):
            vb[i].wall = WALLS[bc["wall"]]
            for q, key in enumerate(("vx", "vy", "vz")):
                if key in bc:
                    vb[i].mask |= 1 << q
                    vb[i].value[q] = float(bc[key])
        keep.append(vb)
        d.n_velocity_bcs = len(self.velocityBCs)
        d.velocity_bcs = vb
        tb = (WallBC * max(1, len(self.temperatureBCs)))()
        for i, bc in enumerate(self.temperatureBCs):
            tb[i].wall = WALLS[bc["wall"]]
            tb[i].mask = 1
            tb[i].value[0] = float(bc["T"])
        keep.append(tb)
        d.n_temperature_bcs = len(self.temperatureBCs)
        d.temperature_bcs = tb
        self._keep = keep
        return d


@dataclass
class State:
    """Host copy of the step state (element-major tet arrays)."""

    coord: np.ndarray
    velocity: np.ndarray
    stress: np.ndarray
    plastic_strain: np.ndarray
    viscosity: np.ndarray
    temperature: np.ndarray
    force: np.ndarray
    inertial_mass: np.ndarray
    plastic_strain_tensor: np.ndarray = None  # [ne, 10, 6], Drucker-Prager phases

    def __post_init__(self):
        if self.plastic_strain_tensor is None:
            self.plastic_strain_tensor = np.zeros(self.stress.shape)

    @classmethod
    def empty(cls, n_elements: int, n_nodes: int) -> "State":
        z = np.zeros
        return cls(coord=z((n_nodes, 3)), velocity=z((n_nodes, 3)), stress=z((n_elements, NT, 6)),
                   plastic_strain=z((n_elements, NT)), viscosity=z((n_elements, NT)),
                   temperature=z(n_nodes), force=z((n_nodes, 3)), inertial_mass=z(n_nodes),
                   plastic_strain_tensor=z((n_elements, NT, 6)))

    def view(self, fields: Optional[Sequence[str]] = None) -> StateView:
        v = StateView()
        for name, _ in StateView._fields_:
            if fields is None or name in fields:
                setattr(v, name, _dptr(getattr(self, name)))
        return v
