"""The FP64 adjoint (snac_gpu_adjoint) against central finite differences of
forward runs: on the GPU, and on the CPU oracle (the reference gradient from
differencing CPU forward runs).  The run yields (Mohr-Coulomb shear branch)
in part of the mesh and keeps the viscosity inside its clip, so all three
gradients are exercised."""
import numpy as np
import pytest

from oracle.pyoracle import Checker
from snac_b200 import workloads as W
from snac_b200.abi import State
from snac_b200.adjoint import SnacMisfit, adjoint, forward_loss, misfit, top_surface
from snac_b200.context import SnacContext, SnacError

pytestmark = pytest.mark.gpu

NX, NY, NZ = 5, 3, 4
NE = NX * NY * NZ
NSTEPS = 24


def make_cfg(coh, fric, visc, plugin="SnacViscoPlastic"):
    cfg = W.c5_adjoint(NX, NY, NZ, dt=1.0e8, v=0.5 * W.CM_PER_YR * 20, extent=(15.0e3, 6.0e3, 12.0e3),
                       cohesion=(5.0e6, 1.0e6), t_uniform=300.0)
    if plugin == "SnacPlastic":
        m = W.mc_phase(c0=5.0e6, c1=1.0e6)
        cfg.plugin = "SnacPlastic"
        cfg.temperature = False
        cfg.temperatureBCs = []
        cfg.init_temperature = None
        cfg.materials = [m]
    cfg.element_cohesion_scale = np.asarray(coh, dtype=np.float64)
    cfg.element_friction_scale = np.asarray(fric, dtype=np.float64)
    cfg.element_visc_scale = np.asarray(visc, dtype=np.float64)
    return cfg


def base_params(seed=1):
    rng = np.random.default_rng(seed)
    return (1.0 + 0.05 * rng.uniform(-1, 1, NE), 1.0 + 0.05 * rng.uniform(-1, 1, NE),
            1.0 + 0.05 * rng.uniform(-1, 1, NE))


def targets(plugin="SnacViscoPlastic"):
    """Top-surface v_y and topography of a run with smooth +-10 % cohesion
    and viscosity perturbations."""
    pc = 1.0 + W.smooth_field(NX, NY, NZ, 7)
    pv = 1.0 + W.smooth_field(NX, NY, NZ, 8)
    with SnacContext(make_cfg(pc, np.ones(NE), pv, plugin)) as ctx:
        ctx.time_step_zero()
        ctx.step(NSTEPS)
        tv, ty = top_surface(ctx.cfg, ctx.state())
    return tv, ty


def weights(tv, ty):
    # scale the two misfit terms to comparable magnitudes
    return 1.0 / max(1e-30, np.mean(tv ** 2)), 1.0 / (6.0e3 ** 2)


def fd_directional(plugin, p, d, h, tv, ty, wv, wh):
    plus = [x + h * dx for x, dx in zip(p, d)]
    minus = [x - h * dx for x, dx in zip(p, d)]
    mk = lambda c, f, v: make_cfg(c, f, v, plugin)
    lp = forward_loss(mk, *plus, NSTEPS, tv, ty, wv, wh)
    lm = forward_loss(mk, *minus, NSTEPS, tv, ty, wv, wh)
    return (lp - lm) / (2.0 * h)


@pytest.mark.parametrize("plugin", ["SnacViscoPlastic", "SnacPlastic"])
def test_adjoint_matches_finite_differences(plugin):
    tv, ty = targets(plugin)
    wv, wh = weights(tv, ty)
    p = base_params()
    with SnacContext(make_cfg(*p, plugin)) as ctx:
        ctx.time_step_zero()
        r = adjoint(ctx, NSTEPS, tv, ty, wv, wh, checkpoint_every=5)
        end = ctx.state()
        assert np.count_nonzero(end.plastic_strain) > 0  # the shear branch was taken
    # the loss equals a plain forward run's
    l0 = forward_loss(lambda c, f, v: make_cfg(c, f, v, plugin), *p, NSTEPS, tv, ty, wv, wh)
    assert r.loss == l0
    g = [r.grad["cohesion"], r.grad["friction"], r.grad["viscosity"]]
    assert all(np.all(np.isfinite(x)) for x in g)
    rng = np.random.default_rng(3)
    worst = 0.0
    for _ in range(4):
        d = [rng.standard_normal(NE) for _ in range(3)]
        if plugin == "SnacPlastic":
            d[2] = np.zeros(NE)  # no viscosity in the plastic hook
        ad = sum(float(np.dot(a, b)) for a, b in zip(g, d))
        fd = fd_directional(plugin, p, d, 1.0e-6, tv, ty, wv, wh)
        rel = abs(ad - fd) / max(abs(fd), 1e-300)
        worst = max(worst, rel)
        print(f"{plugin}: adjoint {ad:.12e}  fd {fd:.12e}  rel {rel:.2e}")
    assert worst <= 1.0e-5


def test_adjoint_against_cpu_oracle_differences():
    """Reference gradient: central differences of the CPU oracle's forward runs."""
    tv, ty = targets()
    wv, wh = weights(tv, ty)
    p = base_params(2)
    with SnacContext(make_cfg(*p)) as ctx:
        ctx.time_step_zero()
        r = adjoint(ctx, NSTEPS, tv, ty, wv, wh)
    g = [r.grad["cohesion"], r.grad["friction"], r.grad["viscosity"]]

    def cpu_loss(params):
        c = Checker(make_cfg(*params), "port")
        c.time_step_zero()
        c.step(NSTEPS)
        v, y = top_surface(make_cfg(*params), c.state())
        return float(np.sum(wv * (v - tv) ** 2 + wh * (y - ty) ** 2))

    rng = np.random.default_rng(5)
    d = [rng.standard_normal(NE) for _ in range(3)]
    h = 1.0e-6
    fd = (cpu_loss([x + h * dx for x, dx in zip(p, d)]) - cpu_loss([x - h * dx for x, dx in zip(p, d)])) / (2 * h)
    ad = sum(float(np.dot(a, b)) for a, b in zip(g, d))
    print(f"oracle fd {fd:.12e}  adjoint {ad:.12e}")
    assert abs(ad - fd) <= 1.0e-5 * abs(fd)


def test_adjoint_is_reproducible_and_leaves_the_final_state():
    tv, ty = targets()
    p = base_params()
    outs = []
    for _ in range(2):
        with SnacContext(make_cfg(*p)) as ctx:
            ctx.time_step_zero()
            r = adjoint(ctx, NSTEPS, tv, ty, checkpoint_every=7)
            outs.append((r, ctx.state()))
    with SnacContext(make_cfg(*p)) as ctx:
        ctx.time_step_zero()
        ctx.step(NSTEPS)
        plain = ctx.state()
    for k in ("cohesion", "friction", "viscosity"):
        assert np.array_equal(outs[0][0].grad[k], outs[1][0].grad[k])
    for f in ("coord", "velocity", "stress", "plastic_strain"):
        assert np.array_equal(getattr(outs[0][1], f), getattr(plain, f))


def test_checkpoint_interval_does_not_change_the_gradient():
    tv, ty = targets()
    p = base_params()
    res = []
    for k in (1, 4, NSTEPS):
        with SnacContext(make_cfg(*p)) as ctx:
            ctx.time_step_zero()
            res.append(adjoint(ctx, NSTEPS, tv, ty, checkpoint_every=k))
    for r in res[1:]:
        for k in ("cohesion", "friction", "viscosity"):
            assert np.array_equal(r.grad[k], res[0].grad[k])


def test_autograd_function():
    import torch
    tv, ty = targets()
    wv, wh = weights(tv, ty)
    p = base_params()
    coh, fric, visc = (torch.tensor(x, dtype=torch.float64, requires_grad=True) for x in p)
    L = SnacMisfit.apply(coh, fric, visc, make_cfg, NSTEPS, tv, ty, wv, wh)
    (2.0 * L).backward()
    with SnacContext(make_cfg(*p)) as ctx:
        ctx.time_step_zero()
        r = adjoint(ctx, NSTEPS, tv, ty, wv, wh)
    assert float(L) == r.loss
    assert np.array_equal(coh.grad.numpy(), 2.0 * r.grad["cohesion"])
    assert np.array_equal(visc.grad.numpy(), 2.0 * r.grad["viscosity"])


def test_unsupported_physics_is_refused():
    cfg = make_cfg(*base_params())
    cfg.dtType = "dynamic"
    tv = np.zeros((NX + 1) * (NZ + 1))
    with SnacContext(cfg) as ctx:
        ctx.time_step_zero()
        with pytest.raises(SnacError) as e:
            adjoint(ctx, 3, tv, tv)
        assert e.value.code == -9
    # the Drucker-Prager return map (an iteration count that switches with a
    # tolerance test) is not differentiated
    from tests import scenarios as S
    dp = S.constant_dt(S.drucker_prager_small(5, 3, 4), 1.0e8)
    tv = np.zeros((dp.nx + 1) * (dp.nz + 1))
    with SnacContext(dp) as ctx:
        ctx.time_step_zero()
        with pytest.raises(SnacError) as e:
            adjoint(ctx, 3, tv, tv)
        assert e.value.code == -9


# ---- gradients with respect to the entry state, all four hooks --------------------------
#
# FLAC damping multiplies the force by 1 - demf sgn(v) sgn(F): the loss jumps
# wherever a perturbation moves a velocity or force component across zero at
# some step, and central differences across a jump measure jump / 2h, not the
# derivative (the adjoint is exact for the discretisation either way).  The
# state gradients are therefore checked with the damping off (demf = 0),
# where the loss is smooth away from the return map's branch switches, from
# an entry state whose velocities got a seeded random field after time step
# zero (no exact symmetry is left).

# field: (state name, direction scale, step h); the plastic-strain direction
# is relative to each tet's own plastic strain (it must stay on the table)
STATE_FIELDS = {"coordinates": ("coord", 10.0, 1.0e-6), "velocity": ("velocity", 1.0e-9, 1.0e-6),
                "stress": ("stress", 1.0e5, 1.0e-5), "plastic_strain": ("plastic_strain", None, 1.0e-4)}


def state_cfg(plugin):
    """The adjoint workload through one of the four hooks; the elastic and
    Maxwell hooks take no per-element scales."""
    base = "SnacPlastic" if plugin == "SnacPlastic" else "SnacViscoPlastic"
    cfg = make_cfg(*base_params(), base)
    cfg.demf = 0.0
    if plugin in ("SnacElastic", "SnacMaxwell"):
        cfg.plugin = plugin
        cfg.element_cohesion_scale = cfg.element_friction_scale = cfg.element_visc_scale = None
    return cfg


WARM = 6  # steps before the entry state, so that yielded tets carry plastic strain
FIELDS = ["coord", "velocity", "stress", "plastic_strain"]


def enter(ctx, field=None, delta=None):
    """Time step zero, a seeded velocity field, WARM steps, then the state
    uploaded again (with `delta` added to one field)."""
    ctx.time_step_zero()
    s = ctx.state()
    rng = np.random.default_rng(17)
    s.velocity += 0.05 * W.CM_PER_YR * rng.standard_normal(s.velocity.shape)
    ctx.set_state(s, ["velocity"])
    ctx.step(WARM)
    s = ctx.state()
    if field is not None:
        a = getattr(s, field)
        a += delta.reshape(a.shape)
    ctx.set_state(s, FIELDS)
    return s


def state_targets(cfg):
    with SnacContext(cfg) as ctx:
        enter(ctx)
        ctx.step(NSTEPS)
        v, y = top_surface(cfg, ctx.state())
    rng = np.random.default_rng(11)
    return v * (1.0 + 0.2 * rng.uniform(-1, 1, v.size)), y + 5.0 * rng.uniform(-1, 1, y.size)


def loss_from_perturbed(cfg, field, delta, tv, ty, wv, wh):
    with SnacContext(cfg) as ctx:
        enter(ctx, field, delta)
        ctx.step(NSTEPS)
        return misfit(ctx, tv, ty, wv, wh)


@pytest.mark.parametrize("plugin", ["SnacElastic", "SnacMaxwell", "SnacPlastic", "SnacViscoPlastic"])
def test_state_gradients_match_finite_differences(plugin):
    cfg = state_cfg(plugin)
    tv, ty = state_targets(cfg)
    wv, wh = weights(tv, ty)
    with SnacContext(cfg) as ctx:
        s0 = enter(ctx)
        r = adjoint(ctx, NSTEPS, tv, ty, wv, wh, checkpoint_every=5, state=True)
        end = ctx.state()
    eps0 = s0.plastic_strain.reshape(-1)
    if plugin in ("SnacElastic", "SnacMaxwell"):
        for k in ("cohesion", "friction", "viscosity", "plastic_strain"):
            assert not np.any(r.grad[k]), k  # no scale or plastic strain enters these hooks
    else:
        assert np.count_nonzero(end.plastic_strain) > 0  # the shear branch was taken
    if plugin in ("SnacMaxwell", "SnacViscoPlastic"):
        assert np.any(end.viscosity > 1.0e19) and np.any(end.viscosity < 1.0e24)
    rng = np.random.default_rng(13)
    fields = [k for k in STATE_FIELDS if k != "plastic_strain" or plugin in ("SnacPlastic", "SnacViscoPlastic")]
    for k in fields:
        name, scale, h = STATE_FIELDS[k]
        g = r.grad[k].reshape(-1)
        assert np.all(np.isfinite(g)) and np.any(g != 0.0), k
        if k == "plastic_strain":
            assert np.count_nonzero(eps0) > 0
            d = eps0 * rng.standard_normal(g.size)  # zero where no plastic strain yet
        else:
            d = scale * rng.standard_normal(g.size)
        ad = float(np.dot(g, d))
        # central differences at three steps: their truncation error grows with
        # the step and their rounding error as its inverse, so the differences
        # disagree among themselves where either dominates, while an error of
        # the adjoint shows as a disagreement with all three
        rels = []
        for hh in (4.0 * h, h, 0.25 * h):
            fd = (loss_from_perturbed(cfg, name, hh * d, tv, ty, wv, wh) -
                  loss_from_perturbed(cfg, name, -hh * d, tv, ty, wv, wh)) / (2.0 * hh)
            rels.append(abs(ad - fd) / max(abs(fd), 1e-300))
            print(f"{plugin} {k}: adjoint {ad:.12e}  fd {fd:.12e}  rel {rels[-1]:.2e}  (h {hh:g})")
        assert min(rels) <= 1.0e-5, (k, ad, rels)


def test_state_gradient_checkpointing_is_exact():
    cfg = state_cfg("SnacMaxwell")
    tv, ty = state_targets(cfg)
    res = []
    for k in (1, 5, NSTEPS):
        with SnacContext(cfg) as ctx:
            enter(ctx)
            res.append(adjoint(ctx, NSTEPS, tv, ty, checkpoint_every=k, state=True))
    for r in res[1:]:
        for k in ("coordinates", "velocity", "stress"):
            assert np.array_equal(r.grad[k], res[0].grad[k]), k
