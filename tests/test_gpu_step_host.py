"""snac_gpu_step_host: one step of a state the host keeps, with the uploads,
the kernels and the downloads overlapped slab by slab, gives the bits of
snac_gpu_upload + snac_gpu_step(1) + snac_gpu_download, for every slab
count and mesh shape, and leaves the handle where those three calls leave
it (graph steps afterwards continue with the same bits)."""
import numpy as np
import pytest
import torch

from snac_b200 import workloads as W
from snac_b200.abi import State
from snac_b200.context import SnacContext, SnacError
from tests import scenarios as S

pytestmark = pytest.mark.gpu

MOVED = ["coord", "velocity", "stress", "plastic_strain", "viscosity"]
ALL = ("coord", "velocity", "stress", "plastic_strain", "viscosity", "temperature", "force", "inertial_mass")


def pinned(s: State, keep: list) -> State:
    """The same arrays in page-locked host memory (the overlapped form)."""
    for f in ALL + ("plastic_strain_tensor",):
        t = torch.from_numpy(np.ascontiguousarray(getattr(s, f))).pin_memory()
        keep.append(t)
        setattr(s, f, t.numpy())
    return s


def nudge(s: State, i: int):
    """A host-side change between steps, so that the upload is what the step reads."""
    s.velocity *= 1.0 + 1.0e-3 * (i + 1)
    s.stress[::7] *= 1.0 - 1.0e-4
    s.temperature[::5] += 0.5


def assert_same(x: State, y: State, fields=MOVED):
    for f in fields:
        a, b = getattr(x, f), getattr(y, f)
        assert np.array_equal(a, b), (f, int(np.sum(a != b)))


def assert_same_scalars(a: SnacContext, b: SnacContext):
    p, q = a.scalars(), b.scalars()
    assert (p.dt, p.min_length_scale, p.vmax, p.time_step, p.current_time) == \
           (q.dt, q.min_length_scale, q.vmax, q.time_step, q.current_time)


def compare(cfg, warm, steps, chunks, use_pinned=True, after=4):
    moved = MOVED + (["temperature"] if cfg.temperature else [])
    a, b = SnacContext(cfg), SnacContext(cfg)
    keep = []
    try:
        for x in (a, b):
            x.time_step_zero()
            x.step(warm)
        sa = a.state()
        sb = b.state()
        if use_pinned:
            sb = pinned(sb, keep)
        for i in range(steps):
            nudge(sa, i)
            nudge(sb, i)
            a.set_state(sa, moved)            # the three calls
            a.step(1)
            a.state(sa)
            b.step_host(sb, sb, chunks=chunks)  # in place
            assert_same(sa, sb, moved)
            assert_same_scalars(a, b)
        a.step(after)
        b.step(after)
        assert_same(a.state(), b.state(), ALL)
        assert_same_scalars(a, b)
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("chunks", [0, 1, 3, 16, 64])
@pytest.mark.parametrize("case", ["elastic", "plastic", "plastic_phases", "lithostatic", "winkler", "traction",
                                  "viscoplastic", "maxwell", "drucker_prager", "density"])
def test_same_bits_as_upload_step_download(case, chunks):
    """with temperature (visco-plastic, Maxwell, Drucker-Prager, two-phase
    density) the heat flux and temperature update run as slab stages too"""
    make, _ = S.CASES[case]
    compare(make(), 6, 5, chunks)


def test_topography_diffusion_takes_the_three_calls():
    """a wavefront over the whole top surface: the same call, the same bits"""
    make, _ = S.CASES["topo"]
    compare(make(), 4, 3, 0)


@pytest.mark.parametrize("shape", [(1, 1, 1), (1, 3, 1), (2, 1, 5), (3, 2, 1), (5, 3, 7), (13, 5, 11)])
@pytest.mark.parametrize("make", [S.elastic_small, S.plastic_small, S.viscoplastic_small])
def test_ragged_meshes_and_empty_slabs(make, shape):
    """hex counts that split no k-layer into whole element blocks, and more
    slabs than the mesh has blocks (empty slabs launch nothing)"""
    for chunks in (2, 7, 64):
        compare(make(*shape), 3, 4, chunks, after=2)


def test_pageable_host_arrays():
    make, _ = S.CASES["plastic"]
    compare(make(), 6, 3, 0, use_pinned=False)


def test_separate_in_and_out_arrays():
    """`in` is only read, `out` receives the result; arrays that change from
    call to call (here the two buffers swap roles) give the same bits"""
    cfg = S.plastic_small()
    a, b = SnacContext(cfg), SnacContext(cfg)
    keep = []
    for x in (a, b):
        x.time_step_zero()
        x.step(8)
    src = pinned(a.state(), keep)
    dst = pinned(State.empty(b.ne, b.nn), keep)
    for _ in range(5):
        before = {f: getattr(src, f).copy() for f in MOVED}
        b.step_host(src, dst)
        a.set_state(src, MOVED)
        a.step(1)
        ref = a.state()
        assert_same(ref, dst)
        for f in MOVED:
            assert np.array_equal(getattr(src, f), before[f]), f
        src, dst = dst, src
    a.close()
    b.close()


def test_full_size_plastic_model():
    """the 64 x 32(y) x 64 Mohr-Coulomb model at the default slab count"""
    compare(W.c2_plastic(), 3, 3, 0, after=3)


def test_full_size_viscoplastic_temperature_model():
    """the 128 x 64(y) x 128 visco-plastic model with temperature"""
    compare(W.c3_viscoplastic(), 2, 2, 0, after=2)


def test_refuses_bad_arguments():
    with SnacContext(S.elastic_small()) as ctx:
        s = ctx.state()
        with pytest.raises(SnacError) as e:
            ctx.step_host(s, s)  # before step zero
        assert e.value.code == -10
        ctx.time_step_zero()
        for chunks in (-1, 65):
            with pytest.raises(SnacError) as e:
                ctx.step_host(s, s, chunks=chunks)
            assert e.value.code == -1
        ctx.step_host(s, s, chunks=64)


def test_non_finite_state_is_reported_as_by_the_three_calls():
    """a NaN uploaded with the state: the status snac_gpu_upload +
    snac_gpu_step + snac_gpu_download give, with an element or node index
    (the first of the tets or nodes that see it to report; the fault is
    made on the host, nothing faults on the GPU)"""
    make, _ = S.CASES["plastic"]
    errs = []
    for host_step in (False, True):
        with SnacContext(make()) as ctx:
            ctx.time_step_zero()
            ctx.step(3)
            s = ctx.state()
            s.velocity[17, 2] = np.nan
            with pytest.raises(SnacError) as e:
                if host_step:
                    ctx.step_host(s, s, chunks=4)
                else:
                    ctx.set_state(s, MOVED)
                    ctx.step(1)
                    ctx.state(s)
            errs.append((e.value.code, e.value.index))
    assert errs[0][0] == errs[1][0] == -4  # ENAN
    assert errs[0][1] >= 0 and errs[1][1] >= 0
