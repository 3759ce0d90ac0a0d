"""The SnacCuda plugin (snac_b200/plugin): a Snac_Context built by the
reference's own hot-path sources (compiled against oracle/refshim), into
which the plugin is loaded the way StGermain's PluginLoader loads it
(PluginLoader.c:359-370) and which is then driven through its entry points
the way AbstractContext drives it.

CPU: the plugin finds its _Register by name, replaces exactly the loop
entry points (EntryPoint_Replace, EntryPoint.c:735), fills the descriptor
from the context (per-node conditions found by applying the context's own
VariableConditions), and copies the state between the context's arrays of
structs and the library's element-major arrays and back bit for bit.

GPU: the context stepped through the plugin's hooks ends where the
reference sources stepped on the CPU end: bitwise for elastic and
constant-angle plastic physics, within the visco-plastic tolerance (1e-6)
where the device evaluates the Arrhenius viscosity.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle
from snac_b200.abi import Desc, State
from tests import scenarios as S

pytestmark = pytest.mark.skipif(not pyoracle.available("plugin_host") and not pyoracle.available("reference"),
                                reason="reference sources not compiled (no SNAC tree)")

FIELDS = ("coord", "velocity", "stress", "plastic_strain", "viscosity", "temperature", "force", "inertial_mass")
_DP = C.POINTER(C.c_double)


class CudaContext(C.Structure):
    """SnacCuda_Context (snac_b200/plugin/SnacCuda.h)."""
    _fields_ = [("gpu", C.c_void_p), ("constitutive", C.c_int), ("temperature", C.c_int), ("druckerPrager", C.c_int),
                ("plasticElement", C.c_uint), ("viscoPlasticElement", C.c_uint), ("maxwellElement", C.c_uint),
                ("temperatureNode", C.c_uint), ("temperatureContext", C.c_uint),
                ("ne", C.c_longlong), ("nn", C.c_longlong),
                ("coord", _DP), ("velocity", _DP), ("stress", _DP), ("plasticStrain", _DP), ("viscosity", _DP),
                ("temperature_", _DP), ("force", _DP), ("inertialMass", _DP), ("plasticStrainTensor", _DP)]


class DescStore(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("materials", "elementMaterial", "initStress", "initVelocity",
                                          "initTemperature", "velocityBCMask", "velocityBCValue",
                                          "temperatureBCMask", "temperatureBCValue", "dpMaxIterations",
                                          "dpTolerance", "cohesionScale", "frictionScale", "viscScale")]


def host(cfg):
    h = pyoracle.PluginHost(cfg)
    assert h.load_plugin("SnacCuda") == 0
    return h


def plugin_fn(h, name, *argtypes, restype=None):
    f = getattr(h.lib, name)
    f.argtypes = list(argtypes)
    f.restype = restype
    return f


def cuda_ext(h):
    return CudaContext.from_address(h.extension_ptr("SnacCuda"))


def test_plugin_replaces_the_loop_entry_points():
    h = host(S.plastic_small())
    assert h.hooks("Context_Initialise") == ["SnacCuda"]            # was SnacTimeStepZero
    assert h.hooks("Context_Solve") == ["SnacCuda_BeginStep", "SnacSolve"]
    assert h.hooks("Context_Sync") == ["SnacCuda"]                  # was SnacSync
    assert h.hooks("Context_Dump")[0] == "SnacCuda_SyncHost"
    for ep in ("Snac_EP_CalcStresses", "Snac_EP_LoopNodesMomentum", "Snac_EP_LoopElementsMomentum"):
        assert h.hooks(ep) == ["SnacCuda"]                          # was "default"
    assert h.hooks("Snac_EP_Constitutive") == ["SnacPlastic"]       # the physics plugin stays
    assert h.hooks("Snac_EP_LoopElementsEnergy") == []              # no temperature plugin: untouched
    t = host(S.viscoplastic_small())
    assert t.hooks("Snac_EP_LoopElementsEnergy") == ["SnacCuda"]
    assert t.hooks("Snac_EP_LoopNodesEnergy") == ["SnacCuda"]


def test_unknown_plugin_is_refused():
    h = pyoracle.PluginHost(S.elastic_small())
    assert h.load_plugin("SnacNoSuchPlugin") != 0


@pytest.mark.parametrize("case", ["plastic", "viscoplastic", "maxwell", "winkler", "drucker_prager"])
def test_pack_unpack_round_trip_bitwise(case):
    """State of a context stepped by the reference sources -> the library's
    arrays (pack) equal its own element-major view; wiping the context and
    unpacking gives every field back to the last bit."""
    make, _ = S.CASES[case]
    cfg = make()
    h = host(cfg)
    assert h.time_step_zero() == 0 and h.step(7) == 0
    want = h.state()
    ctx, ext = h.context_ptr(), h.extension_ptr("SnacCuda")
    assert plugin_fn(h, "SnacCuda_Inspect", C.c_void_p, C.c_void_p, restype=C.c_int)(ctx, ext) == 0
    plugin_fn(h, "SnacCuda_Pack", C.c_void_p, C.c_void_p)(ctx, ext)
    cx = cuda_ext(h)
    ne, nn = cfg.n_elements, cfg.n_nodes
    assert (cx.ne, cx.nn) == (ne, nn)
    packed = {"coord": (cx.coord, nn * 3), "velocity": (cx.velocity, nn * 3), "stress": (cx.stress, ne * 60),
              "plastic_strain": (cx.plasticStrain, ne * 10), "viscosity": (cx.viscosity, ne * 10),
              "temperature": (cx.temperature_, nn), "plastic_strain_tensor": (cx.plasticStrainTensor, ne * 60)}
    assert bool(cx.plasticStrainTensor) == (case == "drucker_prager")
    if case == "drucker_prager":
        assert np.count_nonzero(want.plastic_strain_tensor) > 0
    for f, (p, n) in packed.items():
        if p:
            assert np.array_equal(np.ctypeslib.as_array(p, (n,)), getattr(want, f).reshape(-1)), f
    # the download side: force and inertial mass come back too
    np.ctypeslib.as_array(cx.force, (nn * 3,))[:] = want.force.reshape(-1)
    np.ctypeslib.as_array(cx.inertialMass, (nn,))[:] = want.inertial_mass
    zero = State.empty(ne, nn)
    h.set_state(zero)  # wipe what the unpack writes
    plugin_fn(h, "SnacCuda_Unpack", C.c_void_p, C.c_void_p)(ctx, ext)
    got = h.state()
    for f in FIELDS + ("plastic_strain_tensor",):
        if f in ("plastic_strain",) and cfg.plugin not in ("SnacPlastic", "SnacViscoPlastic"):
            continue
        assert np.array_equal(getattr(got, f), getattr(want, f)), f


def _wall_mask(cfg, wall):
    nnx, nny, nnz = cfg.nx + 1, cfg.ny + 1, cfg.nz + 1
    k, j, i = np.meshgrid(np.arange(nnz), np.arange(nny), np.arange(nnx), indexing="ij")
    i, j, k = i.reshape(-1), j.reshape(-1), k.reshape(-1)
    return {"back": k == 0, "left": i == 0, "bottom": j == 0, "right": i == nnx - 1, "top": j == nny - 1,
            "front": k == nnz - 1, "all": np.ones_like(i, bool)}[wall]


@pytest.mark.parametrize("case", ["elastic", "lithostatic", "viscoplastic", "traction", "plastic_phases"])
def test_fill_desc_from_the_context(case):
    """The descriptor the plugin builds from the context: mesh, phases, the
    state after the ICs, and the conditions resolved per node, last VC
    winning, as the configuration's walls say."""
    make, _ = S.CASES[case]
    cfg = make()
    h = host(cfg)
    ctx, ext = h.context_ptr(), h.extension_ptr("SnacCuda")
    assert plugin_fn(h, "SnacCuda_Inspect", C.c_void_p, C.c_void_p, restype=C.c_int)(ctx, ext) == 0
    d, st = Desc(), DescStore()
    fill = plugin_fn(h, "SnacCuda_FillDesc", C.c_void_p, C.c_void_p, C.POINTER(Desc), C.POINTER(DescStore),
                     restype=C.c_int)
    assert fill(ctx, ext, C.byref(d), C.byref(st)) == 0
    try:
        ne, nn = cfg.n_elements, cfg.n_nodes
        ref = cfg.desc()
        assert (d.nx, d.ny, d.nz) == (cfg.nx, cfg.ny, cfg.nz)
        assert d.constitutive == ref.constitutive and d.temperature == ref.temperature
        assert d.dt_type == ref.dt_type and d.gravity == ref.gravity and d.demf == ref.demf
        assert d.winkler == ref.winkler and d.traction_bc == ref.traction_bc and d.hydrostatic_ic == 0
        state = h.state()  # the context after its ICs
        assert np.array_equal(np.ctypeslib.as_array(d.init_stress, (ne * 60,)), state.stress.reshape(-1))
        assert np.array_equal(np.ctypeslib.as_array(d.node_coords, (nn * 3,)), state.coord.reshape(-1))
        # conditions: last VC wins per component
        mask = np.zeros(nn, np.uint8)
        val = np.zeros((nn, 3))
        for bc in cfg.velocityBCs:
            w = _wall_mask(cfg, bc["wall"])
            for q, key in enumerate(("vx", "vy", "vz")):
                if key in bc:
                    mask[w] |= 1 << q
                    val[w, q] = bc[key]
        got_mask = np.ctypeslib.as_array(d.node_velocity_bc_mask, (nn,))
        got_val = np.ctypeslib.as_array(d.node_velocity_bc_value, (nn * 3,)).reshape(nn, 3)
        assert np.array_equal(got_mask, mask)
        fixed = np.stack([(mask >> q) & 1 for q in range(3)], axis=1).astype(bool)
        assert np.array_equal(got_val[fixed], val[fixed])
        if cfg.temperature:
            tmask = np.zeros(nn, np.uint8)
            for bc in cfg.temperatureBCs:
                tmask[_wall_mask(cfg, bc["wall"])] = 1
            assert np.array_equal(np.ctypeslib.as_array(d.node_temperature_bc_mask, (nn,)), tmask)
        if cfg.hydrostatic_ic:
            assert d.pisos != 0.0 and d.rzbo == cfg.min[1]
        if cfg.element_cohesion_scale is not None:
            # one phase per element in the context, grouped back into scaled base phases:
            # each element's cohesion table is reproduced to the bit by base x scale
            assert 1 <= d.n_materials <= 32 and d.element_cohesion_scale
            cs = np.ctypeslib.as_array(d.element_cohesion_scale, (ne,))
            em = np.ctypeslib.as_array(d.element_material, (ne,))
            for e in range(ne):
                base = d.materials[int(em[e])]
                for i in range(base.nsegments + 1):
                    src = cfg.materials[cfg.element_material[e] if cfg.element_material is not None else 0]
                    want = src[f"cohesion{i}"] * cfg.element_cohesion_scale[e]
                    assert base.cohesion[i] * cs[e] == want
        # the probe leaves the context's velocities as they were
        assert np.array_equal(h.state().velocity, state.velocity)
    finally:
        plugin_fn(h, "SnacCuda_FreeDescStore", C.POINTER(DescStore))(C.byref(st))


def relerr(a, b):
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / den) if den > 0 else float(np.max(np.abs(a - b)))


@pytest.mark.gpu
@pytest.mark.parametrize("case, tol", [("elastic", 0.0), ("plastic", 0.0), ("plastic_phases", 0.0),
                                       ("lithostatic", 0.0), ("winkler", 0.0), ("traction", 0.0), ("topo", 0.0),
                                       ("viscoplastic", 1e-6), ("maxwell", 1e-9), ("drucker_prager", 1e-6)])
def test_context_driven_through_the_plugin(case, tol):
    """60 steps of a Snac_Context through the plugin's hooks (step zero,
    then Dt / Solve / Sync per step, then Dump) against the compiled
    reference sources stepping the same configuration on the CPU."""
    make, _ = S.CASES[case]
    cfg = make()
    steps = 60
    h = host(cfg)
    assert h.initialise() == 0, h.last_error()
    assert h.host_step(steps // 2) == 0, h.last_error()
    assert h.dump() == 0                                   # device -> context
    mid = h.state()
    assert h.host_step(steps - steps // 2) == 0, h.last_error()
    assert h.dump() == 0
    got = h.state()
    ref = pyoracle.Checker(cfg, "reference")
    assert ref.time_step_zero() == 0
    ref.step(steps // 2)
    ref_mid = ref.state()
    ref.step(steps - steps // 2)
    want = ref.state()
    fields = list(FIELDS) + ["plastic_strain_tensor"]
    for a, b in ((mid, ref_mid), (got, want)):
        for f in fields:
            x, y = getattr(a, f), getattr(b, f)
            if tol == 0.0:
                assert np.array_equal(x, y), (case, f, relerr(x, y))
            else:
                assert relerr(x, y) <= tol, (case, f, relerr(x, y))
    assert h.scalars().dt == ref.scalars().dt or tol > 0


def test_unrelated_phases_beyond_the_table_are_refused():
    """Forty phases that differ in their elastic moduli are not scaled copies
    of a base phase: the descriptor cannot express them and is refused."""
    from snac_b200 import workloads as W
    cfg = S.plastic_small()
    cfg.element_cohesion_scale = None
    base = cfg.materials[0]
    cfg.materials = [dict(base, mu=base["mu"] * (1.0 + 0.01 * p)) for p in range(40)]
    cfg.element_material = (np.arange(cfg.n_elements) % 40).astype(np.int32)
    h = host(cfg)
    ctx, ext = h.context_ptr(), h.extension_ptr("SnacCuda")
    assert plugin_fn(h, "SnacCuda_Inspect", C.c_void_p, C.c_void_p, restype=C.c_int)(ctx, ext) == 0
    d, st = Desc(), DescStore()
    fill = plugin_fn(h, "SnacCuda_FillDesc", C.c_void_p, C.c_void_p, C.POINTER(Desc), C.POINTER(DescStore),
                     restype=C.c_int)
    try:
        assert fill(ctx, ext, C.byref(d), C.byref(st)) == -9  # SNAC_GPU_ENOTSUP
    finally:
        plugin_fn(h, "SnacCuda_FreeDescStore", C.POINTER(DescStore))(C.byref(st))
