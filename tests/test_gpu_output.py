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


def expected_dump(ck, plastic, visc, temperature):
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
    if temperature:
        rec["temperature"] = s.temperature.astype(np.float32)
    return rec


def expected_checkpoint(ck, plastic, visc, temperature):
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
    if temperature:
        rec["temperatureCP"] = s.temperature.astype(np.float32)
    return rec


def run(tmp_path, case, nsteps=7, dump_every=3, cp_every=4):
    cfg = S.CASES[case][0]()
    plastic = cfg.plugin in ("SnacPlastic", "SnacViscoPlastic")
    visc = cfg.plugin == "SnacViscoPlastic"
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
                for k, v in expected_dump(ck, plastic, visc, cfg.temperature).items():
                    expect.setdefault(k, []).append(v)
                lines_dump.append(line)
            if ts == nsteps or ts % cp_every == 0:
                for k, v in expected_checkpoint(ck, plastic, visc, cfg.temperature).items():
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


def test_write_output_needs_open():
    from snac_b200.context import SnacError
    with SnacContext(S.CASES["elastic"][0]()) as g:
        g.time_step_zero()
        g.step(1)
        with pytest.raises(SnacError):
            g.write_output()
