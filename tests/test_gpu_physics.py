"""Artificial viscosity and optically thin radiation on the GPU against the C++ oracle (GPU required).

fluid/ArtificialViscosity.m (Neumann-Richtmyer, Caramana-Shashkov-Whalen) adds a viscous pressure to
the 'totsnd' pressure of both wFluidFlux.m stages; fluid/Radiation.m's optically thin sink is applied by
source.m:30 after each timestep's flux, with the strength Radiation.initialize takes from the initial
state.  Tolerances (relative L1 per variable, FP64): 1e-12 after one sweep, 1e-10 after 100 iterations;
the mixed form (FP32 state) against the FP64 oracle at 2e-5.  Strengths are run_Debug.m's: viscosity
0.1 (linear) / 0.25 (quadratic), radiation exponent 0.5 and initialMaximum 0.1.
"""
import numpy as np
import pytest

from imogen_b200 import ImogenBatch, ImogenError, ImogenRun, problems
from oracle import cpp_oracle
from tests.parity import errors, make_pair, smooth_state

pytestmark = pytest.mark.gpu

VISC = ("neumann_richtmyer", "caramana_shashkov_whalen")


def _settings(grid, bc="circ", **kw):
    s = dict(grid=grid, dgrid=tuple(1 / g for g in grid), gamma=5 / 3, cfl=0.35, bc=bc, magnet=True,
             time_max=1e5, iter_max=10 ** 6, visc_linear=0.1, visc_quadratic=0.25, rad_exponent=0.5,
             rad_initial_maximum=0.1)
    s.update(kw)
    return s


def _compressive(grid, seed=4):
    """smooth_state with the momentum scaled by 4 (and E raised to keep the pressure): strong
    converging regions where both viscosities act."""
    rho, mom, ener, mag = smooth_state(grid, seed=seed, mhd=True)
    mom4 = 4 * mom
    return rho, mom4, ener + 0.5 * (mom4 ** 2 - mom ** 2).sum(0) / rho, mag


def _check(o, g, tol, what):
    e = errors(g.state(), o.state())
    bad = {k: v for k, v in e.items() if not (v <= tol)}
    assert not bad, f"{what}: relative L1 above {tol}: {bad}"


@pytest.mark.parametrize("viscosity", VISC)
@pytest.mark.parametrize("grid,bc", [((64, 32, 1), "circ"), ((64, 32, 1), "const"), ((32, 16, 16), "circ"),
                                     ((32, 16, 16), "const")])
def test_viscosity_one_sweep_per_direction(viscosity, grid, bc):
    s = _settings(grid, bc, viscosity=viscosity)
    o, g = make_pair(s, _compressive(grid))
    o.time_update(1)
    g.time.update(1, sync=True)
    for X in (1, 2, 3):
        if grid[X - 1] < 3:
            continue
        o.relaxing_fluid(X)
        g.relaxing_fluid(X)
        _check(o, g, 1e-12, f"{viscosity} {bc} {grid} after the sweep along {X}")
    g.close()


@pytest.mark.parametrize("viscosity", VISC)
@pytest.mark.parametrize("bc", ["circ", "const"])
def test_viscosity_100_iterations(viscosity, bc):
    grid = (64, 32, 1)
    s = _settings(grid, bc, viscosity=viscosity)
    st = _compressive(grid)
    o, g = make_pair(s, st)
    assert o.run(100) == 100 and g.run(100) == 100
    _check(o, g, 1e-10, f"{viscosity} {bc} after 100 iterations")
    # the viscosity is doing something: the inviscid oracle run differs
    ref = cpp_oracle.Sim(**problems.oracle_kwargs(_settings(grid, bc)))
    ref.set_state(*st)
    ref.run(100)
    d = errors(o.state(), ref.state())
    assert max(d.values()) > 1e-6, d
    g.close()


def test_viscosity_3d_30_iterations():
    grid = (32, 16, 16)
    for viscosity in VISC:
        o, g = make_pair(_settings(grid, "circ", viscosity=viscosity), _compressive(grid, seed=9))
        assert o.run(30) == 30 and g.run(30) == 30
        _check(o, g, 1e-10, f"{viscosity} 3-D after 30 iterations")
        g.close()


@pytest.mark.parametrize("viscosity", VISC)
def test_viscosity_mixed_form(viscosity):
    grid = (64, 32, 1)
    o, g = make_pair(_settings(grid, "circ", viscosity=viscosity), _compressive(grid), precision="mixed")
    o.run(100)
    g.run(100)
    _check(o, g, 2e-5, f"{viscosity} mixed form after 100 iterations")
    g.close()


@pytest.mark.parametrize("bc", ["circ", "trans", "wall"])
@pytest.mark.parametrize("update_mode", [1, 0])
def test_radiation_100_iterations(bc, update_mode):
    grid = (48, 40, 1)
    s = _settings(grid, bc, radiation="optically_thin", update_mode=update_mode)
    o, g = make_pair(s, smooth_state(grid, seed=2, mhd=True))
    assert o.rad_strength > 0
    assert g.radiation_strength == pytest.approx(o.rad_strength, rel=1e-13)
    o.iterate()
    g.iterate()
    _check(o, g, 1e-12, f"radiation {bc} mode {update_mode} after one iteration")
    o.run(99)
    g.run(99)
    assert g.time.time == pytest.approx(o.time, rel=1e-12)
    _check(o, g, 1e-10, f"radiation {bc} mode {update_mode} after 100 iterations")
    g.close()


def test_source_step_by_step():
    """time.update, flux and source called one at a time (imogen.m:62-67) match the oracle's."""
    grid = (48, 40, 1)
    o, g = make_pair(_settings(grid, radiation="optically_thin"), smooth_state(grid, seed=6, mhd=True))
    for i, order in ((1, 1), (2, -1)):
        o.time_update(i)
        g.time.update(i, sync=True)
        o.flux(order)
        g.flux(order)
        o.source()
        g.source()
        _check(o, g, 1e-12, f"after source of timestep {i}")
    g.close()


def test_viscosity_and_radiation_together_mixed_and_fp64():
    grid = (64, 32, 1)
    for precision, tol in (("fp64", 1e-10), ("mixed", 2e-5)):
        s = _settings(grid, "const", viscosity="caramana_shashkov_whalen", radiation="optically_thin")
        o, g = make_pair(s, _compressive(grid, seed=8), precision=precision)
        o.run(50)
        g.run(50)
        _check(o, g, tol, f"CSW + radiation {precision} after 50 iterations")
        g.close()


def test_autotune_keeps_segment_tilings_with_viscosity():
    grid = (64, 32, 1)
    r = ImogenRun(**_settings(grid, viscosity="neumann_richtmyer"))
    r.set_state(*_compressive(grid))
    t = r.autotune(trials=1)["fluid"]
    for d in (1, 2):
        assert t[d][6] == 1, t
    with pytest.raises(ImogenError):   # a pencil-tile tiling has no viscous exchanges
        r.set_tiling(1, (1, 64, 1, 64, 1, 1, 0))
    r.close()


def test_physics_contexts_do_not_join_batches():
    grid = (64, 32, 1)
    for extra in (dict(viscosity="neumann_richtmyer"), dict(radiation="optically_thin")):
        r = ImogenRun(**_settings(grid, **extra))
        r.set_state(*_compressive(grid))
        with pytest.raises(ImogenError):
            ImogenBatch([r])
        r.close()
