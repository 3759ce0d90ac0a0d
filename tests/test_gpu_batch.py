"""Batched ensembles on the GPU, through the C ABI.

A batch launches every kernel type once per step over all models; each
model's results must be the single-model results to the last bit (and so
the oracle's, which the single-model path matches), whatever the launch
shape, and whether the batch runs batched or model by model.
"""
import numpy as np
import pytest

from oracle.pyoracle import Checker
from snac_b200 import workloads as W
from snac_b200.batch import SnacBatch, autotune
from snac_b200.context import SnacContext, SnacError

pytestmark = pytest.mark.gpu

FIELDS = ("coord", "velocity", "stress", "plastic_strain", "viscosity", "temperature", "force", "inertial_mass")


def small_ensemble(n=6, seed=11):
    return W.c4_ensemble(n, seed=seed, xz=(3, 7), y=(2, 5))


def assert_same(sa, sb, what):
    for f in FIELDS:
        x, y = getattr(sa, f), getattr(sb, f)
        assert np.array_equal(x, y), (what, f, int(np.sum(x != y)))


def singles(cfgs, steps):
    out = []
    for cfg in cfgs:
        with SnacContext(cfg) as g:
            g.time_step_zero()
            g.step(steps)
            out.append((g.state(), g.scalars().dt))
    return out


def test_batch_equals_single_models_bitwise():
    cfgs = small_ensemble()
    ref = singles(cfgs, 7)
    with SnacBatch(cfgs) as b:
        b.time_step_zero()
        b.step(3)
        b.step(4)
        for i, m in enumerate(b.models):
            assert_same(m.state(), ref[i][0], f"model {i}")
            assert m.scalars().dt == ref[i][1]
            assert m.scalars().time_step == 7


def test_batch_against_oracle():
    cfgs = small_ensemble(4, seed=5)
    with SnacBatch(cfgs) as b:
        b.time_step_zero()
        b.step(5)
        for i, cfg in enumerate(cfgs):
            c = Checker(cfg, "port")
            c.time_step_zero()
            c.step(5)
            sg, sc = b.models[i].state(), c.state()
            if cfg.plugin == "SnacPlastic":  # constant friction angle: bitwise
                assert_same(sg, sc, f"model {i}")
            else:  # device log/exp in the viscosity: plastic tolerance
                for f in ("coord", "velocity", "stress", "temperature"):
                    x, y = getattr(sg, f), getattr(sc, f)
                    assert np.max(np.abs(x - y)) <= 1e-6 * np.max(np.abs(y)), (i, f)


@pytest.mark.parametrize("tuning", [
    {"node_threads": 64, "minls_threads": 256},
    {"elem_blocks_per_sm": 2, "node_blocks_per_sm": 1},
    {"steps_per_graph": 3, "order": 1},
    {"steps_per_graph": 1, "node_threads": 256, "elem_blocks_per_sm": 16},
    {"split_classes": 0, "steps_per_graph": 2},
    {"split_classes": 1, "elem_blocks_per_sm": 3},
])
def test_launch_shape_does_not_change_results(tuning):
    cfgs = small_ensemble(5, seed=3)
    ref = singles(cfgs, 8)
    with SnacBatch(cfgs) as b:
        b.tuning = tuning
        assert all(b.tuning[k] == v for k, v in tuning.items())
        b.time_step_zero()
        b.step(8)
        for i, m in enumerate(b.models):
            assert_same(m.state(), ref[i][0], f"model {i} {tuning}")


def test_batch_with_per_element_phases_bitwise():
    """A two-phase model (per-element phase table, density coupling) batched
    with one-phase models: the phase-table path of the batch kernels gives
    the single-model bits."""
    from tests import scenarios as S
    cfgs = [S.CASES["density"][0](), S.CASES["plastic"][0](), S.CASES["viscoplastic"][0]()]
    ref = singles(cfgs, 6)
    with SnacBatch(cfgs) as b:
        b.time_step_zero()
        b.step(6)
        for i, m in enumerate(b.models):
            assert_same(m.state(), ref[i][0], f"model {i}")


def test_step_each_equals_batched():
    cfgs = small_ensemble(5, seed=8)
    with SnacBatch(cfgs) as a, SnacBatch(cfgs) as b:
        a.time_step_zero()
        b.time_step_zero()
        a.step(6)
        b.step_each(6)
        for i in range(len(cfgs)):
            assert_same(a.models[i].state(), b.models[i].state(), f"model {i}")
        # mixing the two forms keeps the models in step
        a.step_each(2)
        b.step(2)
        for i in range(len(cfgs)):
            assert_same(a.models[i].state(), b.models[i].state(), f"model {i} mixed")


def test_one_model_read_mid_run():
    """Downloading one model applies its deferred element update; the batch
    flushes the others before the next step and the results stay exact."""
    cfgs = small_ensemble(4, seed=9)
    ref = singles(cfgs, 6)
    with SnacBatch(cfgs) as b:
        b.time_step_zero()
        b.step(3)
        b.models[2].state()
        b.step(3)
        for i, m in enumerate(b.models):
            assert_same(m.state(), ref[i][0], f"model {i}")


def test_model_stepped_alone_is_refused():
    cfgs = small_ensemble(3, seed=2)
    with SnacBatch(cfgs) as b:
        b.time_step_zero()
        b.models[1].step(1)
        with pytest.raises(SnacError) as e:
            b.step(1)
        assert e.value.index == 1


def test_error_names_the_model():
    cfgs = small_ensemble(3, seed=4)
    with SnacBatch(cfgs) as b:
        b.time_step_zero()
        b.step(1)
        s = b.models[2].state()
        s.velocity[5] = np.nan
        b.models[2].set_state(s, ["velocity"])
        with pytest.raises(SnacError) as e:
            b.step(2)
        assert e.value.index == 2


def test_batch_before_step_zero_is_refused():
    with SnacBatch(small_ensemble(2)) as b:
        with pytest.raises(SnacError):
            b.step(1)


def test_invalid_tuning_is_refused():
    with SnacBatch(small_ensemble(2)) as b:
        with pytest.raises(SnacError):
            b.tuning = {"node_threads": 48}
        with pytest.raises(SnacError):
            b.tuning = {"steps_per_graph": 0}


def test_autotune_applies_and_caches(tmp_path):
    cfgs = small_ensemble(4, seed=6)
    cache = str(tmp_path / "tune.json")
    with SnacBatch(cfgs) as b:
        t = autotune(b, steps=3, cache_path=cache)
        assert b.tuning == t
        b.time_step_zero()
        b.step(4)
        ref = singles(cfgs, 4)
        for i, m in enumerate(b.models):
            assert_same(m.state(), ref[i][0], f"model {i}")
    with SnacBatch(cfgs) as b2:
        assert autotune(b2, cache_path=cache) == t
