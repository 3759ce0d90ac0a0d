"""Small seeded cases shared by the CPU and GPU parity tests.

Every case is a reduced copy of a benchmark configuration (same physics,
fewer elements, and loads strong enough that the plastic branch is taken
within a few hundred steps) or one of the reference's own test fixtures.
"""
import numpy as np

from snac_b200 import workloads as W
from snac_b200.abi import F32, SnacConfig


def elastic_small(nx=8, ny=4, nz=8):
    return W.c1_elastic(nx, ny, nz)


def plastic_small(nx=8, ny=4, nz=8, active=True):
    """C2 physics; with active=True: no gravity and a weak, fast-softening
    phase, so that tension/shear yielding starts within ~10 steps."""
    cfg = W.c2_plastic(nx, ny, nz)
    if active:
        cfg.gravity = 0.0
        cfg.hydrostatic_ic = False
        cfg.materials = [W.mc_phase(c0=2.0e5, c1=2.0e4, eps1=0.001)]
    return cfg


def viscoplastic_small(nx=8, ny=4, nz=8, active=True):
    cfg = W.c3_viscoplastic(nx, ny, nz, extent=(100.0e3, 20.0e3, 100.0e3), sigma=5.0e3)
    if active:
        cfg.gravity = 0.0
        cfg.hydrostatic_ic = False
        m = W.vp_phase()
        m.update(W.mc_phase(c0=2.0e5, c1=2.0e4, eps1=0.001, flat_tail=1.0e3))
        cfg.materials = [m]
    return cfg


def drucker_prager_small(nx=8, ny=4, nz=8, maxiterations=1):
    """The yielding visco-plastic case with the Drucker-Prager criterion
    (viscoplastic/Constitutive.c:372-518); maxiterations > 1 takes the
    iterated return map."""
    cfg = viscoplastic_small(nx, ny, nz)
    for m in cfg.materials:
        m["yieldcriterion"] = "druckerprager"
        m["maxiterations"] = maxiterations
        m["constitutivetolerance"] = 1.0e-3
    return cfg


def maxwell_small(nx=6, ny=4, nz=6):
    cfg = W.c3_viscoplastic(nx, ny, nz, extent=(100.0e3, 20.0e3, 100.0e3), sigma=5.0e3)
    cfg.plugin = "SnacMaxwell"
    return cfg


def lithostatic_small(nx=8, ny=4, nz=8):
    """C2 exactly (gravity, lithostatic IC, per-element cohesion), small."""
    return W.c2_plastic(nx, ny, nz)


def winkler_small(nx=8, ny=4, nz=8):
    """The lithostatic plastic case with the SnacWinklerForce plugin holding the
    bottom up instead of a roller: no vy condition on the bottom wall."""
    cfg = W.c2_plastic(nx, ny, nz)
    cfg.winkler = True
    cfg.velocityBCs = [bc for bc in cfg.velocityBCs if bc["wall"] != "bottom"]
    return cfg


def traction_small(nx=8, ny=4, nz=8):
    """Elastic, the right wall free in x and pushed by the SnacTractionBC stress."""
    cfg = W.c1_elastic(nx, ny, nz)
    cfg.traction_bc = True
    cfg.velocityBCs = [bc for bc in cfg.velocityBCs if bc["wall"] != "right"]
    return cfg


def topo_small(nx=8, ny=4, nz=8, kappa=0.5):
    """The lithostatic plastic case with surface-topography diffusion on."""
    cfg = W.c2_plastic(nx, ny, nz)
    cfg.topo_kappa = kappa
    return cfg


def two_phase_density(nx=6, ny=4, nz=6):
    """Two phases with thermal expansion and compressibility (per-tet density
    path) under gravity, with temperature and thermal stress."""
    cfg = W.c3_viscoplastic(nx, ny, nz, extent=(60.0e3, 20.0e3, 60.0e3), sigma=5.0e3)
    a = W.vp_phase()
    b = W.vp_phase(density=3000.0)
    for m in (a, b):
        m["alpha"] = 3.0e-5
        m["beta"] = 1.0e-11
    cfg.materials = [a, b]
    rng = np.random.default_rng(11)
    cfg.element_material = rng.integers(0, 2, cfg.n_elements).astype(np.int32)
    cfg.computeThermalStress = True
    return cfg


def plastic_two_phase(nx=8, ny=4, nz=8):
    """The yielding plastic case with two Mohr-Coulomb phases (different
    cohesion and softening) assigned per element: the phase-table path."""
    cfg = plastic_small(nx, ny, nz)
    cfg.materials = [W.mc_phase(c0=2.0e5, c1=2.0e4, eps1=0.001), W.mc_phase(c0=4.0e5, c1=1.0e5, eps1=0.002)]
    rng = np.random.default_rng(13)
    cfg.element_material = rng.integers(0, 2, cfg.n_elements).astype(np.int32)
    return cfg


def constant_dt(cfg: SnacConfig, dt: float) -> SnacConfig:
    cfg.dtType = "constant"
    cfg.timeStep = dt
    return cfg


def cube100(velocity=(0.0, 0.0, 0.0)) -> SnacConfig:
    """The 100 m mesh of the libSnac force/geometry tests: 4x4x4 nodes over
    [0,300] x [-300,0] x [0,300], gravity 9.81, density 2700, uniform velocity."""
    D = {"density": 2700.0, "alpha": 0.0, "beta": 0.0, "lambda": F32(3.0e10), "mu": F32(3.0e10)}
    cfg = SnacConfig(nx=3, ny=3, nz=3, min=(0.0, -300.0, 0.0), max=(300.0, 0.0, 300.0),
                     dtType="dynamic", timeStep=0.0, strain_inert=F32(1.0e-5), gravity=9.81,
                     demf=F32(0.8), plugin="SnacElastic", materials=[D], velocityBCs=[])
    v = np.zeros((cfg.n_nodes, 3))
    v[:] = velocity
    cfg.init_velocity = v.reshape(-1)
    return cfg


def pull_test_10(ctx):
    """The 10-iteration loop of Snac/libSnac/tests/testUpdateNode-velocity-4-4-4.c:
    element update, strain rate + stress, node force + update, with the
    context's timeStep left at 0."""
    for _ in range(10):
        ctx.loop_elements_momentum()
        ctx.calc_stresses()
        ctx.loop_nodes_momentum()


CASES = {
    "elastic": (elastic_small, 60),
    "plastic": (plastic_small, 120),
    "viscoplastic": (viscoplastic_small, 120),
    "maxwell": (maxwell_small, 60),
    "lithostatic": (lithostatic_small, 60),
    "winkler": (winkler_small, 60),
    "traction": (traction_small, 60),
    "topo": (topo_small, 60),
    "density": (two_phase_density, 40),
    "plastic_phases": (plastic_two_phase, 120),
    "drucker_prager": (drucker_prager_small, 120),
    "drucker_prager_iterated": (lambda: drucker_prager_small(maxiterations=4), 120),
}
