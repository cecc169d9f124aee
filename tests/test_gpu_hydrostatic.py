"""The hydrostatic-tank configuration (2.0 x 1.0 m water, dx = 0.002 m,
500,000 fluid particles, 3 wall layers, 2,000 steps) against its analytic
answer: pressure p = rho0 g (H - y), with the water kept in the tank and its
volume conserved.

The pressure profile is judged as the mean pressure of depth bins two
spacings thick, away from the side walls, against rho0 g (H - y_bin):
per-particle pressures of weakly-compressible SPH carry acoustic noise of a
few percent that the profile averages out.  Bound: 3 % of rho0 g H for the
textbook WCSPH profile in FP64 and with FP32 pair arithmetic."""
import numpy as np
import pytest

from uph_b200 import deck as D

pytestmark = pytest.mark.gpu

RHO0, G = 1000.0, 9.81


def _conservation(state, init, nf, width):
    """(fluid particles outside the tank interior, relative drift of the
    water volume sum m / rho).  Particle masses never change, so mass is
    conserved exactly iff no fluid particle is lost: the count is what
    shows it.  The volume sum shows the mean density holding."""
    x, y = state["Position"][:nf, 0], state["Position"][:nf, 1]
    outside = int(np.count_nonzero(~((x > 0.0) & (x < width) & (y > 0.0) & np.isfinite(x) & np.isfinite(y))))
    v0 = float(np.sum(init["mass"][:nf] / init["density"][:nf]))
    v1 = float(np.sum(state["mass"][:nf] / state["density"][:nf]))
    return outside, abs(v1 - v0) / v0


def _binned_error(state, nf, depth, width, dx):
    y = state["Position"][:nf, 1]
    x = state["Position"][:nf, 0]
    p = state["DynamicPressure"][:nf]
    keep = (x > 5 * dx) & (x < width - 5 * dx)
    bins = np.arange(0.0, depth + 2 * dx, 2 * dx)
    idx = np.digitize(y[keep], bins)
    worst = 0.0
    for b in range(1, len(bins)):
        m = idx == b
        if m.sum() < 10:
            continue
        yc = y[keep][m].mean()
        worst = max(worst, abs(p[keep][m].mean() - RHO0 * G * (depth - yc)))
    return worst / (RHO0 * G * depth)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32_pair"])
def test_hydrostatic_tank_matches_rho_g_h(precision):
    from uph_b200.sim import Simulation

    width, depth, dx = 2.0, 1.0, 0.002
    deck = D.hydrostatic_tank(width=width, depth=depth, dx=dx, layers=3)
    assert deck.n_fluid == 500_000
    init = deck.initial_state()
    with Simulation.from_deck(deck, profile=1, precision=precision) as s:
        s.step(2000)
        st = s.download()
        stats = s.stats()
    nf = deck.n_fluid
    err = _binned_error(st, nf, depth, width, dx)
    assert err <= 0.03, f"pressure profile off by {100 * err:.2f} % of rho0 g H"
    outside, dvol = _conservation(st, init, nf, width)
    print(f"precision {precision}: profile error {100 * err:.3f} % of rho0 g H, volume drift {dvol:.2e}")
    assert outside == 0, f"{outside} fluid particles left the tank"
    assert dvol < 1e-3, f"water volume drifted by {dvol:.2e}"
    assert stats["max_abs_density_error"] < 0.01
    # the water stays put: no particle moved more than a spacing
    drift = np.abs(st["Position"][:nf] - init["Position"][:nf]).max()
    assert drift < dx, f"max drift {drift:.2e} m"


def test_hydrostatic_tank_ref_profile_is_stable():
    """The reference's own formulation on the same tank (its diffusion and
    fluctuation terms make the profile converge more slowly): bounded
    velocities, the profile within 10 % of rho0 g H, no fluid lost and the
    water volume held."""
    from uph_b200.sim import Simulation

    width, depth, dx = 2.0, 1.0, 0.002
    deck = D.hydrostatic_tank(width=width, depth=depth, dx=dx, layers=3)
    with Simulation.from_deck(deck, profile=0) as s:
        s.step(2000)
        st = s.download()
    nf = deck.n_fluid
    err = _binned_error(st, nf, depth, width, dx)
    outside, dvol = _conservation(st, deck.initial_state(), nf, width)
    print(f"REF: profile error {100 * err:.3f} % of rho0 g H, volume drift {dvol:.2e}, "
          f"max |v| {np.abs(st['Velocity'][:nf]).max():.3e}")
    assert np.abs(st["Velocity"][:nf]).max() < 0.5
    assert err <= 0.10
    assert outside == 0, f"{outside} fluid particles left the tank"
    assert dvol < 1e-3, f"water volume drifted by {dvol:.2e}"
