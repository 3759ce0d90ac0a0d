"""Host-side logic of the batched ensembles (no GPU): the ensemble workload,
the autotuner's search and its cache key."""
import numpy as np

from snac_b200 import workloads as W
from snac_b200.abi import BatchTuning
from snac_b200.batch import SEARCH_SPACE, batch_signature, search


def test_ensemble_workload_shapes():
    cfgs = W.c4_ensemble()
    assert len(cfgs) == 256
    for c in cfgs:
        assert 8 <= c.nx <= 48 and 8 <= c.nz <= 48 and 4 <= c.ny <= 24
    plugins = {c.plugin for c in cfgs}
    assert plugins == {"SnacPlastic", "SnacViscoPlastic"}
    coh = np.array([c.materials[0]["cohesion0"] for c in cfgs])
    phi = np.array([c.materials[0]["frictionAngle0"] for c in cfgs])
    assert coh.min() >= 10.0e6 and coh.max() <= 60.0e6
    assert phi.min() >= 15.0 and phi.max() <= 35.0
    visc = np.array([c.materials[0]["refvisc"] for c in cfgs if c.plugin == "SnacViscoPlastic"])
    assert visc.min() >= 1.0e20 and visc.max() <= 1.0e23
    # seeded: the same list twice
    again = W.c4_ensemble()
    assert [(c.nx, c.ny, c.nz) for c in cfgs] == [(c.nx, c.ny, c.nz) for c in again]


def test_signature_depends_on_shapes_only():
    a = W.c4_ensemble(6, seed=1, xz=(3, 6), y=(2, 4))
    b = W.c4_ensemble(6, seed=1, xz=(3, 6), y=(2, 4))
    c = W.c4_ensemble(6, seed=2, xz=(3, 6), y=(2, 4))
    assert batch_signature(a) == batch_signature(b)
    assert batch_signature(a) != batch_signature(c)
    assert batch_signature(a).startswith("6:")


def test_search_finds_the_separable_minimum():
    # a cost that is separable in the knobs: coordinate descent must find its minimum
    target = {"steps_per_graph": 16, "elem_blocks_per_sm": 8, "node_threads": 256,
              "node_blocks_per_sm": 0, "minls_threads": 64, "order": 1, "split_classes": 0}
    calls = []

    def measure(t):
        calls.append(dict(t))
        return 1.0 + sum(abs(SEARCH_SPACE[k].index(t[k]) - SEARCH_SPACE[k].index(target[k])) for k in target)

    start = {"steps_per_graph": 1, "elem_blocks_per_sm": 0, "node_threads": 128,
             "node_blocks_per_sm": 8, "minls_threads": 128, "order": 0, "split_classes": 1}
    best, ms, tried = search(measure, start)
    assert best == target and ms == 1.0
    assert len(tried) == len(calls) == 1 + sum(len(v) - 1 for v in SEARCH_SPACE.values())


def test_tuning_struct_round_trip():
    d = {"node_threads": 64, "minls_threads": 256, "elem_blocks_per_sm": 4, "node_blocks_per_sm": 0,
         "steps_per_graph": 8, "order": 1, "split_classes": 0}
    assert BatchTuning.from_dict(d).as_dict() == d
