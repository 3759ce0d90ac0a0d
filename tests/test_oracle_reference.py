"""The plain-C restatement against the reference's own hot-path sources,
compiled here from the SNAC tree against oracle/refshim (oracle/_ref).
Every field must agree to the last bit, for every rheology and IC path."""
import os

import numpy as np
import pytest

from oracle import pyoracle
from tests import scenarios as S

REF_TREE = pyoracle.snac_tree()


def _reference_available():
    if pyoracle.available("reference"):
        return True
    if os.path.isdir(REF_TREE):
        try:
            pyoracle.build("reference")
            return True
        except Exception:
            return False
    return False


pytestmark = pytest.mark.skipif(not _reference_available(), reason="reference checker not built (no SNAC tree)")

FIELDS = ("coord", "velocity", "stress", "plastic_strain", "viscosity", "temperature", "force", "inertial_mass")


@pytest.mark.parametrize("case", sorted(S.CASES))
def test_restatement_is_bitwise_equal_to_reference(case):
    make, steps = S.CASES[case]
    cfg = make()
    a = pyoracle.Checker(cfg, "port")
    b = pyoracle.Checker(cfg, "reference")
    assert a.time_step_zero() == 0 and b.time_step_zero() == 0
    for _ in range(2):
        a.step(steps // 2)
        b.step(steps // 2)
        sa, sb = a.state(), b.state()
        for f in FIELDS:
            x, y = getattr(sa, f), getattr(sb, f)
            assert np.array_equal(x, y), (case, f, np.max(np.abs(x - y)))
        assert a.scalars().dt == b.scalars().dt
        assert a.scalars().min_length_scale == b.scalars().min_length_scale
        assert a.scalars().current_time == b.scalars().current_time
        # element scalars of the dump files: strain rate, stress, hydroPressure, aps
        ea, eb = a.element_scalars(), b.element_scalars()
        for k in ("strain_rate", "stress", "hydro_pressure", "aps", "volume"):
            assert np.array_equal(ea[k], eb[k]), (case, k)


def test_plastic_case_actually_yields():
    a = pyoracle.Checker(S.plastic_small(), "port")
    a.time_step_zero()
    a.step(S.CASES["plastic"][1])
    assert np.count_nonzero(a.state().plastic_strain) > 100


def test_pull_test_bitwise():
    from snac_b200 import workloads as W
    a = pyoracle.Checker(W.libsnac_unit_cube(), "port")
    b = pyoracle.Checker(W.libsnac_unit_cube(), "reference")
    a.time_step_zero()
    b.time_step_zero()
    S.pull_test_10(a)
    S.pull_test_10(b)
    assert np.array_equal(a.state().velocity, b.state().velocity)


@pytest.mark.parametrize("case", ["plastic", "viscoplastic", "winkler", "traction", "topo", "elastic"])
def test_threaded_reference_is_bitwise_equal_to_serial(case):
    """The all-cores CPU baseline (libsnacref_mt.so: the same reference
    sources, element and node loops split over threads) gives the serial
    build's bits; the topography case keeps its node update in node order."""
    if not pyoracle.available("reference_mt"):
        pytest.skip("threaded reference checker not built")
    make, steps = S.CASES[case]
    cfg = make()
    a = pyoracle.Checker(cfg, "reference")
    b = pyoracle.Checker(cfg, "reference_mt", threads=3)
    assert b.threads == 3
    assert a.time_step_zero() == 0 and b.time_step_zero() == 0
    a.step(steps)
    b.step(steps)
    sa, sb = a.state(), b.state()
    for f in FIELDS:
        assert np.array_equal(getattr(sa, f), getattr(sb, f)), (case, f)
    assert a.scalars().dt == b.scalars().dt


@pytest.mark.parametrize("make", [S.elastic_small, S.viscoplastic_small])
def test_verbatim_bc_search_gives_the_same_bits(make):
    """The boundary conditions applied by StGermain's linear index search
    (the reference's cost) and by the per-node mask give the same state."""
    cfg = make(6, 4, 6)
    a, b = pyoracle.Checker(cfg, "reference"), pyoracle.Checker(cfg, "reference")
    b.set_verbatim_bc(True)
    for c in (a, b):
        assert c.time_step_zero() == 0
        assert c.step(25) == 0
    sa, sb = a.state(), b.state()
    for f in ("coord", "velocity", "stress", "plastic_strain", "temperature"):
        assert np.array_equal(getattr(sa, f), getattr(sb, f)), f
