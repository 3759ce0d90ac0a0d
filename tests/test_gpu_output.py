"""Dump and checkpoint files (snac_gpu_output_open / snac_gpu_write_output)
against the same records formed from the CPU oracle's state with the
reference's conversions (Context.c:1311-1531: float32 casts, the
float-accumulated volume-weighted stress tensor; the plugins' Output.c)."""
import os

import numpy as np
import pytest

from oracle.pyoracle import Checker
from snac_b200.context import SnacContext
from tests import scenarios as S

pytestmark = pytest.mark.gpu


def stress_tensor(stress, vol):
    """Context.c:1469-1490 in float: totalVolume and the six sums are floats."""
    ne = stress.shape[0]
    tv = np.zeros(ne, np.float32)
    for t in range(10):
        tv = (tv.astype(np.float64) + vol[:, t]).astype(np.float32)
    sv = np.zeros((ne, 6), np.float32)
    for t in range(10):
        for a in range(6):
            term = stress[:, t, a] * vol[:, t] / tv.astype(np.float64)
            sv[:, a] = (sv[:, a].astype(np.float64) + term).astype(np.float32)
    return sv


def maxwell_log_visc(visc):
    """maxwell/Output.c:57-118: the tet mean accumulated in a float, log10 when positive."""
    v = np.zeros(visc.shape[0], np.float32)
    for t in range(10):
        v = (v.astype(np.float64) + visc[:, t] / 10).astype(np.float32)
    out = v.copy()
    pos = v > 0
    out[pos] = np.log10(v[pos].astype(np.float64)).astype(np.float32)
    return out


def expected_dump(ck, plastic, visc, temperature, maxwell=False):
    s = ck.state()
    el = ck.element_scalars()
    vol, _, _ = ck.geometry()
    rec = {
        "strainRate": el["strain_rate"].astype(np.float32),
        "stress": el["stress"].astype(np.float32),
        "hydroPressure": el["hydro_pressure"].astype(np.float32),
        "phaseIndex": np.zeros(ck.ne, np.int32),
        "coord": s.coord.astype(np.float32).reshape(-1),
        "vel": s.velocity.astype(np.float32).reshape(-1),
        "force": s.force.astype(np.float32).reshape(-1),
        "stressTensor": stress_tensor(s.stress, vol).reshape(-1),
    }
    if plastic:
        rec["plStrain"] = el["aps"].astype(np.float32)
    if visc:
        rec["viscosity"] = np.log10(np.sum(s.viscosity / 10.0, axis=1)).astype(np.float32)
    if maxwell:
        rec["viscosity"] = maxwell_log_visc(s.viscosity)
    if temperature:
        rec["temperature"] = s.temperature.astype(np.float32)
    return rec


def expected_checkpoint(ck, plastic, visc, temperature, maxwell=False):
    s = ck.state()
    rec = {
        "phaseIndexCP": np.zeros(ck.ne, np.int32),
        "coordCP": s.coord.astype(np.float32).reshape(-1),
        "velCP": s.velocity.astype(np.float32).reshape(-1),
        "stressTensorCP": s.stress.astype(np.float32).reshape(-1),
    }
    if plastic:
        rec["plStrainCP"] = s.plastic_strain.astype(np.float32).reshape(-1)
    if visc:
        rec["viscosityCP"] = np.log10(s.viscosity).astype(np.float32).reshape(-1)
    if maxwell:
        rec["viscosityCP"] = maxwell_log_visc(s.viscosity)
    if temperature:
        rec["temperatureCP"] = s.temperature.astype(np.float32)
    return rec


def run(tmp_path, case, nsteps=7, dump_every=3, cp_every=4):
    cfg = S.CASES[case][0]()
    plastic = cfg.plugin in ("SnacPlastic", "SnacViscoPlastic")
    visc = cfg.plugin == "SnacViscoPlastic"
    maxwell = cfg.plugin == "SnacMaxwell"
    out = str(tmp_path)
    expect = {}
    lines_dump, lines_cp = [], []
    ck = Checker(cfg, "port")
    ck.time_step_zero()
    with SnacContext(cfg) as g:
        g.time_step_zero()
        g.output_open(out, 0, dump_every, cp_every, nsteps)
        for ts in range(1, nsteps + 1):
            g.step(1)
            g.write_output()
            ck.step(1)
            sc = ck.scalars()
            line = "%16u %16g %16g\n" % (sc.time_step, sc.current_time, sc.dt)
            if ts == 1 or ts % dump_every == 0:
                for k, v in expected_dump(ck, plastic, visc, cfg.temperature, maxwell).items():
                    expect.setdefault(k, []).append(v)
                lines_dump.append(line)
            if ts == nsteps or ts % cp_every == 0:
                for k, v in expected_checkpoint(ck, plastic, visc, cfg.temperature, maxwell).items():
                    expect.setdefault(k, []).append(v)
                lines_cp.append(line)
        g.output_close()
    return out, expect, lines_dump, lines_cp


@pytest.mark.parametrize("case", ["plastic", "elastic"])
def test_output_files_bitwise(tmp_path, case):
    out, expect, lines_dump, lines_cp = run(tmp_path, case)
    for name, recs in expect.items():
        want = np.concatenate(recs)
        got = np.fromfile(os.path.join(out, f"{name}.0"), dtype=want.dtype)
        assert got.shape == want.shape, name
        assert np.array_equal(got, want), (name, int(np.sum(got != want)))
    assert open(os.path.join(out, "timeStep.0")).read() == "".join(lines_dump)
    assert open(os.path.join(out, "checkpointTimeStep.0")).read() == "".join(lines_cp)
    sim = open(os.path.join(out, "sim.0")).read().split("\n")[0].split()
    cfg = S.CASES[case][0]()
    assert sim == [str(x) for x in (cfg.nx, cfg.ny, cfg.nz, 1, 1, 1, cfg.nx, cfg.ny, cfg.nz)]


def test_output_files_viscoplastic(tmp_path):
    """Device log/exp/log10: the records agree with the oracle's to float rounding."""
    out, expect, _, _ = run(tmp_path, "viscoplastic", nsteps=5, dump_every=2, cp_every=5)
    for name, recs in expect.items():
        want = np.concatenate(recs)
        got = np.fromfile(os.path.join(out, f"{name}.0"), dtype=want.dtype)
        assert got.shape == want.shape, name
        if want.dtype == np.int32:
            assert np.array_equal(got, want), name
        else:
            den = max(float(np.max(np.abs(want))), 1e-300)
            assert float(np.max(np.abs(got.astype(np.float64) - want))) <= 1e-5 * den, name


def test_output_files_maxwell(tmp_path):
    """SnacMaxwell's viscosity.0 / viscosityCP.0 (maxwell/Output.c:57-118): one
    float per element, the tet mean accumulated in a float and its log10;
    device viscosity within the Maxwell bar, so the records agree to float
    rounding."""
    out, expect, _, _ = run(tmp_path, "maxwell", nsteps=6, dump_every=2, cp_every=3)
    cfg = S.CASES["maxwell"][0]()
    for name in ("viscosity", "viscosityCP"):
        want = np.concatenate(expect[name])
        got = np.fromfile(os.path.join(out, f"{name}.0"), dtype=np.float32)
        assert got.shape == want.shape == (len(expect[name]) * cfg.n_elements,), name
        assert float(np.max(np.abs(got.astype(np.float64) - want))) <= 1e-5 * float(np.max(np.abs(want))), name
    for name, recs in expect.items():
        want = np.concatenate(recs)
        got = np.fromfile(os.path.join(out, f"{name}.0"), dtype=want.dtype)
        assert got.shape == want.shape, name


def test_velocity_dump_against_the_reference_golden(tmp_path):
    """Snac/tests/test-basic-velocity-completeForceCalc.vel.0.expected (read as
    text into tests/golden/basic_velocity_vel.npz): the GPU writer's vel.0 of
    the same 12-step elastic run, record for record, at the float32 bar the
    oracle meets against the same golden.  The golden was written by an
    older revision that also dumped step 0; the current one (isTimeToDump,
    Context.c:1534-1541) dumps steps 1..12, which are golden records 1..12."""
    from snac_b200 import workloads as W
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "basic_velocity_vel.npz"))["vel"]
    cfg = W.basic_velocity()
    nsteps = gold.shape[0] - 1
    with SnacContext(cfg) as g:
        g.time_step_zero()
        g.output_open(str(tmp_path), 0, 1, 0, nsteps)
        for _ in range(nsteps):
            g.step(1)
            g.write_output()
        g.output_close()
    vel = np.fromfile(os.path.join(str(tmp_path), "vel.0"), dtype=np.float32).reshape(nsteps, -1, 3)
    for s in range(1, nsteps + 1):
        diff = np.abs(vel[s - 1] - gold[s])
        if s < 2:
            assert np.max(diff) <= 1e-6 * 5e-9, s
        else:  # the edge nodes the older revision treated differently (tests/test_oracle_golden.py)
            bad = diff > 1e-3 * 5e-9
            assert bad.mean() < 0.1, s
            nodes = np.nonzero(bad.any(axis=1))[0]
            i, j, k = nodes % 13, (nodes // 13) % 11, nodes // 143
            on_edge = ((j == 0) | (j == 10)).astype(int) + ((k == 0) | (k == 10)).astype(int) + (i <= 1).astype(int)
            assert np.all(on_edge >= 1), s


def test_write_output_needs_open():
    from snac_b200.context import SnacError
    with SnacContext(S.CASES["elastic"][0]()) as g:
        g.time_step_zero()
        g.step(1)
        with pytest.raises(SnacError):
            g.write_output()
