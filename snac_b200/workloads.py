"""Seeded synthetic workloads in the reference's vocabulary.

No public dataset is involved: every input is generated here, on the host,
from a seed, and the same arrays feed the CUDA path and the CPU checkers.
Axis convention of the reference: I = x, J = y (vertical, gravity on -y,
top = j max), K = z.  Sizes are element (hex) counts.

  c1_elastic       16 x 8(y) x 16 hex over 100 x 30 x 100 km, SnacElastic
  c2_plastic       64 x 32(y) x 64 hex over 200 x 40 x 200 km, SnacPlastic,
                   cohesion 44 -> 4 MPa over plastic strain 0..0.5, phi 30,
                   psi 0, per-element cohesion x (1 + U[-0.05, 0.05]),
                   lithostatic IC, g = 9.81, +-0.5 cm/yr per x face
  c3_viscoplastic  128 x 64(y) x 128 hex over 400 x 100 x 400 km,
                   SnacTemperature + SnacViscoPlastic, geotherm 0 -> 1300 C
                   over the 100 km depth plus a seeded Gaussian anomaly,
                   power law n = 3, A = 1e-16 Pa^-n s^-1, E = 200 kJ/mol
  c4_ensemble      256 independent plastic / visco-plastic models, seeded sizes
  c5_adjoint       config-2 physics with viscosity on 32 x 16(y) x 32 hex
"""
from __future__ import annotations

import math
from typing import Dict, List, Optional

import numpy as np

from .abi import F32, SnacConfig

CM_PER_YR = 0.01 / (365.25 * 86400.0)  # m/s
R_GAS = 8.31448  # viscoplastic/Constitutive.c:117


def roller_box_bcs(v_left: float, v_right: float) -> List[Dict]:
    """x faces pulled, back/front (z) and bottom (y) rollers, free top."""
    return [
        {"wall": "left", "vx": v_left},
        {"wall": "right", "vx": v_right},
        {"wall": "back", "vz": 0.0},
        {"wall": "front", "vz": 0.0},
        {"wall": "bottom", "vy": 0.0},
    ]


def elastic_phase(rho=2700.0, lam=3.0e10, mu=3.0e10) -> Dict:
    return {"density": rho, "alpha": 0.0, "beta": 0.0, "lambda": lam, "mu": mu}


def mc_phase(rho=2700.0, lam=3.0e10, mu=3.0e10, c0=44.0e6, c1=4.0e6, eps1=0.5, phi=30.0, psi=0.0,
             flat_tail: Optional[float] = None) -> Dict:
    """Mohr-Coulomb strain-softening phase: cohesion c0 -> c1 over plastic
    strain 0 -> eps1.  flat_tail appends a constant segment up to that
    plastic strain: the visco-plastic hook has no clamp beyond the table
    (viscoplastic/Constitutive.c:279-304)."""
    d = elastic_phase(rho, lam, mu)
    pts = [(0.0, c0), (eps1, c1)] + ([(flat_tail, c1)] if flat_tail else [])
    d["nsegments"] = len(pts) - 1
    for i, (e, c) in enumerate(pts):
        d[f"plstrain{i}"] = e
        d[f"cohesion{i}"] = c
        d[f"frictionAngle{i}"] = phi
        d[f"dilationAngle{i}"] = psi
    d["ten_off"] = 1.0e10  # above c / tan(phi) everywhere: the cutoff is c / tan(phi)
    return d


def power_law_visc(n=3.0, A=1.0e-16, E=200.0e3, refsrate=1.0e-15, reftemp_c=1300.0) -> Dict:
    """Map eta = 1/2 A^(-1/n) edot^(1/n-1) exp(E/(n R T)) onto the reference's
    form refvisc (srJ2/refsrate)^(1/srexponent-1) exp(H/R (1/T - 1/Tref))
    (viscoplastic/Constitutive.c:206-209): H = E/n, and refvisc is the
    power-law viscosity at (refsrate, reftemp)."""
    tref = reftemp_c + 273.15
    refvisc = 0.5 * A ** (-1.0 / n) * refsrate ** (1.0 / n - 1.0) * math.exp(E / (n * R_GAS * tref))
    return {"srexponent": n, "refsrate": refsrate, "reftemp": reftemp_c, "refvisc": refvisc,
            "activationE": E / n}


def c1_elastic(nx=16, ny=8, nz=16, v=1.0 * CM_PER_YR) -> SnacConfig:
    return SnacConfig(
        nx=nx, ny=ny, nz=nz, min=(0.0, -30.0e3, 0.0), max=(100.0e3, 0.0, 100.0e3),
        dtType="dynamic", timeStep=0.0, strain_inert=1.0e-5, gravity=0.0, demf=0.8,
        plugin="SnacElastic", materials=[elastic_phase()], velocityBCs=roller_box_bcs(-v, v))


def c2_plastic(nx=64, ny=32, nz=64, seed=2, v=0.5 * CM_PER_YR, extent=(200.0e3, 40.0e3, 200.0e3)) -> SnacConfig:
    rng = np.random.default_rng(seed)
    ne = nx * ny * nz
    return SnacConfig(
        nx=nx, ny=ny, nz=nz, min=(0.0, -extent[1], 0.0), max=(extent[0], 0.0, extent[2]),
        dtType="dynamic", timeStep=0.0, strain_inert=1.0e-5, gravity=9.81, demf=0.8,
        plugin="SnacPlastic", hydrostatic_ic=True, materials=[mc_phase()],
        element_cohesion_scale=1.0 + rng.uniform(-0.05, 0.05, ne),
        velocityBCs=roller_box_bcs(-v, v))


def geotherm(cfg: SnacConfig, t_top=0.0, t_bottom=1300.0, anomaly=200.0, sigma=2.0e3, seed=3) -> np.ndarray:
    """Linear geotherm over the depth plus one Gaussian anomaly at a seeded spot."""
    rng = np.random.default_rng(seed)
    nnx, nny, nnz = cfg.nx + 1, cfg.ny + 1, cfg.nz + 1
    x = cfg.min[0] + (cfg.max[0] - cfg.min[0]) * (np.arange(nnx) / (nnx - 1))
    y = cfg.min[1] + (cfg.max[1] - cfg.min[1]) * (np.arange(nny) / (nny - 1))
    z = cfg.min[2] + (cfg.max[2] - cfg.min[2]) * (np.arange(nnz) / (nnz - 1))
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    depth = (cfg.max[1] - Y) / (cfg.max[1] - cfg.min[1])
    T = t_top + (t_bottom - t_top) * depth
    c = (rng.uniform(0.3, 0.7) * (cfg.max[0] - cfg.min[0]) + cfg.min[0],
         cfg.min[1] + rng.uniform(0.3, 0.7) * (cfg.max[1] - cfg.min[1]),
         rng.uniform(0.3, 0.7) * (cfg.max[2] - cfg.min[2]) + cfg.min[2])
    r2 = (X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2
    T = T + anomaly * np.exp(-0.5 * r2 / sigma ** 2)
    return np.ascontiguousarray(T.reshape(-1))


def vp_phase(eps_tail=1.0e3, **kw) -> Dict:
    d = mc_phase(flat_tail=eps_tail)
    d.update(power_law_visc())
    d.update({"vis_min": 1.0e19, "vis_max": 1.0e24, "thermal_conduct": 3.0, "heatCapacity": 1000.0})
    d.update(kw)
    return d


def c3_viscoplastic(nx=128, ny=64, nz=128, seed=3, v=0.5 * CM_PER_YR,
                    extent=(400.0e3, 100.0e3, 400.0e3), sigma=2.0e3) -> SnacConfig:
    cfg = SnacConfig(
        nx=nx, ny=ny, nz=nz, min=(0.0, -extent[1], 0.0), max=(extent[0], 0.0, extent[2]),
        dtType="dynamic", timeStep=0.0, strain_inert=1.0e-5, gravity=9.81, demf=0.8,
        plugin="SnacViscoPlastic", temperature=True, hydrostatic_ic=True, materials=[vp_phase()],
        velocityBCs=roller_box_bcs(-v, v),
        temperatureBCs=[{"wall": "top", "T": 0.0}, {"wall": "bottom", "T": 1300.0}])
    cfg.init_temperature = geotherm(cfg, sigma=sigma, seed=seed)
    return cfg


def c5_adjoint(nx=32, ny=16, nz=32, seed=5, dt=2.0e7, v=0.5 * CM_PER_YR, t_uniform=600.0,
               extent=(100.0e3, 20.0e3, 100.0e3), cohesion=(44.0e6, 4.0e6)) -> SnacConfig:
    """Adjoint workload: the plastic workload's physics (Mohr-Coulomb
    strain softening, lithostatic IC, gravity, extension) through the
    visco-plastic hook so that a viscosity field exists, with a constant dt
    and a uniform, fixed temperature (zero conductivity).  Per-element
    cohesion, friction and viscosity scales start at 1."""
    cfg = c3_viscoplastic(nx, ny, nz, seed=seed, v=v, extent=extent)
    m = vp_phase(thermal_conduct=0.0)
    m.update(mc_phase(c0=cohesion[0], c1=cohesion[1], flat_tail=1.0e3))
    m.update({k: val for k, val in vp_phase(thermal_conduct=0.0).items() if k not in m})
    cfg.materials = [m]
    cfg.temperatureBCs = [{"wall": "top", "T": t_uniform}, {"wall": "bottom", "T": t_uniform}]
    cfg.init_temperature = np.full(cfg.n_nodes, t_uniform)
    ne = nx * ny * nz
    cfg.element_cohesion_scale = np.ones(ne)
    cfg.element_friction_scale = np.ones(ne)
    cfg.element_visc_scale = np.ones(ne)
    cfg.dtType = "constant"
    cfg.timeStep = dt
    return cfg


def smooth_field(nx, ny, nz, seed, amplitude=0.1) -> np.ndarray:
    """Seeded smooth perturbation in [-amplitude, amplitude] per element (a
    few low-wavenumber sine modes), for targets of the adjoint workload."""
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    f = np.zeros((nz, ny, nx))
    for _ in range(4):
        a, b, c = rng.integers(1, 3, 3)
        ph = rng.uniform(0, 2 * math.pi, 3)
        f += np.sin(math.pi * a * (i + 0.5) / nx + ph[0]) * np.sin(math.pi * b * (j + 0.5) / ny + ph[1]) * \
            np.sin(math.pi * c * (k + 0.5) / nz + ph[2])
    f /= max(1e-30, np.max(np.abs(f)))
    return amplitude * f.reshape(-1)


def ensemble_member(rng: np.random.Generator, plastic: bool, xz=(8, 48), y=(4, 24)) -> SnacConfig:
    nx, ny, nz = int(rng.integers(xz[0], xz[1] + 1)), int(rng.integers(y[0], y[1] + 1)), int(rng.integers(xz[0], xz[1] + 1))
    coh = math.exp(rng.uniform(math.log(10.0e6), math.log(60.0e6)))
    phi = float(rng.uniform(15.0, 35.0))
    refvisc = math.exp(rng.uniform(math.log(1.0e20), math.log(1.0e23)))
    extent = (nx * 3.0e3, ny * 1.5e3, nz * 3.0e3)
    if plastic:
        cfg = c2_plastic(nx, ny, nz, seed=int(rng.integers(1 << 30)), extent=extent)
        cfg.element_cohesion_scale = None
        cfg.materials = [mc_phase(c0=coh, c1=0.1 * coh, phi=phi)]
    else:
        cfg = c3_viscoplastic(nx, ny, nz, seed=int(rng.integers(1 << 30)), extent=extent, sigma=4.0e3)
        m = vp_phase()
        m.update(mc_phase(c0=coh, c1=0.1 * coh, phi=phi, flat_tail=1.0e3))
        m.update({k: v for k, v in vp_phase().items() if k not in m})
        m["refvisc"] = refvisc
        cfg.materials = [m]
    return cfg


def c4_ensemble(n_models=256, seed=4, xz=(8, 48), y=(4, 24)) -> List[SnacConfig]:
    """Batched ensemble: half Mohr-Coulomb plastic, half visco-plastic with a
    geotherm; hex counts drawn per model in [8..48] x [4..24](y) x [8..48]."""
    rng = np.random.default_rng(seed)
    return [ensemble_member(rng, plastic=(i % 2 == 0), xz=xz, y=y) for i in range(n_models)]


# ---- the reference's own test fixtures ------------------------------------------------------

def libsnac_unit_cube() -> SnacConfig:
    """Snac/libSnac/tests/test*-4-4-4.c: 3x3x3 nodes over [0,1] x [-1,0] x [0,1],
    elastic with the dictionary defaults, dtType constant, timeStep 1,
    gravity 0, alpha 0, walls left vx=0 / right vx=0.01 / back,front vz=0 /
    bottom,top vy=0 (testUpdateNode-velocity-4-4-4.c:93-212)."""
    D = {"density": 2700.0, "alpha": 0.0, "beta": 0.0, "lambda": F32(3.0e10), "mu": F32(3.0e10)}
    return SnacConfig(
        nx=2, ny=2, nz=2, min=(F32(0.0), F32(-1.0), F32(0.0)), max=(F32(1.0), F32(0.0), F32(1.0)),
        dtType="constant", timeStep=1.0, strain_inert=F32(1.0e-5), gravity=0.0, demf=F32(0.8),
        plugin="SnacElastic", materials=[D],
        velocityBCs=[{"wall": "left", "vx": 0.0}, {"wall": "right", "vx": 0.01},
                     {"wall": "back", "vz": 0.0}, {"wall": "front", "vz": 0.0},
                     {"wall": "bottom", "vy": 0.0}, {"wall": "top", "vy": 0.0}])


def basic_velocity() -> SnacConfig:
    """Snac/tests/basic-velocity-completeForceCalc.xml: 13x11x11 nodes over
    7500 x 6300 x 6300 m, elastic (defaults), dt = 1e4 constant, demf 0.8,
    right wall fixed, left wall vy = -5e-9."""
    D = {"density": 2700.0, "alpha": 0.0, "beta": 0.0, "lambda": F32(3.0e10), "mu": F32(3.0e10)}
    return SnacConfig(
        nx=12, ny=10, nz=10, min=(0.0, -6300.0, 0.0), max=(7500.0, 0.0, 6300.0),
        dtType="constant", timeStep=10000.0, strain_inert=F32(1.0e-5), gravity=0.0, demf=0.8,
        plugin="SnacElastic", materials=[D],
        velocityBCs=[{"wall": "right", "vx": 0.0, "vy": 0.0, "vz": 0.0}, {"wall": "left", "vy": -5.0e-9}])


def basic_timestep() -> SnacConfig:
    """Snac/tests/basic.xml: 13x13x13 nodes over 7500 m cubed, elastic with the
    dictionary defaults, dtType not given (dynamic), no velocity BCs.  Its
    known answer (test-basic.timeStep.0.expected) is the first dt,
    1.80422e+07 s."""
    D = {"density": 2700.0, "alpha": F32(3.0e-05), "beta": 0.0, "lambda": F32(3.0e10), "mu": F32(3.0e10)}
    return SnacConfig(
        nx=12, ny=12, nz=12, min=(0.0, -7500.0, 0.0), max=(7500.0, 0.0, 7500.0),
        dtType="dynamic", timeStep=0.0, strain_inert=F32(1.0e-5), gravity=0.0, demf=0.8,
        plugin="SnacElastic", materials=[D], velocityBCs=[])
