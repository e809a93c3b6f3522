"""Pins the oracle's velocity damping against the reference's body tests
(crates/bullet-dynamics/src/body.rs, lines cited), in both precisions. Each test's
integrate_velocities is taken through one world step of a lone body with gravity off (the step's
velocity pass; nothing else in the step changes the velocity of a body without contacts).
"""
import numpy as np
import pytest

from oracle_api import ADDITIONAL_DAMPING, OracleWorld

PRECISIONS = ["f32", "f64"]
DT = 1.0 / 60.0


def lone(prec, v, w, flags=0, ld=0.0, ad=0.0):
    o = OracleWorld(prec)
    o.set_gravity((0, 0, 0))
    b = o.add_body(o.sphere(0.5), [0, 0, 0], linvel=v, angvel=w, mass=1.0, flags=flags, lin_damping=ld,
                   ang_damping=ad)
    return o, b


@pytest.mark.parametrize("prec", PRECISIONS)
def test_damping_scales_velocity_exponentially(prec):
    # body.rs:1326-1337: damping 0.5 for 1 s halves both speeds.
    o, b = lone(prec, (10, 0, 0), (0, 0, 20), ld=0.5, ad=0.5)
    for _ in range(60):
        o.step(DT)
    st = o.state()[b]
    assert st[7] == pytest.approx(5.0, abs=1e-4) and st[12] == pytest.approx(10.0, abs=1e-4)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_additional_damping_shrinks_low_speeds(prec):
    # body.rs:1347-1369: below both thresholds the speeds scale by 0.005; above them, or
    # without the flag, nothing happens.
    o, b = lone(prec, (0.05, 0, 0), (0, 0.02, 0), flags=ADDITIONAL_DAMPING)
    o.step(DT)
    st = o.state()[b]
    assert st[7] == pytest.approx(0.05 * 0.005, abs=1e-6) and st[11] == pytest.approx(0.02 * 0.005, abs=1e-6)
    o, b = lone(prec, (1.0, 0, 0), (0, 0.5, 0), flags=ADDITIONAL_DAMPING)
    o.step(DT)
    st = o.state()[b]
    assert st[7] == pytest.approx(1.0, abs=1e-6) and st[11] == pytest.approx(0.5, abs=1e-6)
    o, b = lone(prec, (0.05, 0, 0), (0, 0, 0))
    o.step(DT)
    assert o.state()[b, 7] == pytest.approx(0.05, abs=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_additional_damping_subtract_block_follows_the_upstream_quirk(prec):
    # body.rs:1377-1400: with damping 0.2 both speeds sit under their damping factors and above
    # the 0.005 cut, so each loses exactly 0.005 after the pow pass; a speed under the cut ends
    # at zero.
    pw = (1.0 - 0.2) ** DT
    o, b = lone(prec, (0.04, 0, 0), (0, 0, 0.15), flags=ADDITIONAL_DAMPING, ld=0.2, ad=0.2)
    o.step(DT)
    st = o.state()[b]
    assert st[7] == pytest.approx(0.04 * pw - 0.005, abs=1e-5)
    assert st[12] == pytest.approx(0.15 * pw - 0.005, abs=1e-5)
    o, b = lone(prec, (0.002, 0, 0), (0, 0, 0), flags=ADDITIONAL_DAMPING, ld=0.2, ad=0.2)
    o.step(DT)
    np.testing.assert_array_equal(o.state()[b, 7:10], [0.0, 0.0, 0.0])


@pytest.mark.parametrize("prec", PRECISIONS)
def test_disable_deactivation_never_sleeps(prec):
    # body.rs:1229-1238: ten seconds at rest leave a DisableDeactivation body in that state.
    from oracle_api import DISABLE_DEACTIVATION

    o = OracleWorld(prec)
    o.set_gravity((0, 0, 0))
    b = o.add_body(o.sphere(0.5), [0, 0, 0], mass=1.0, activation=DISABLE_DEACTIVATION)
    for _ in range(600):
        o.step(DT)
    assert int(o.state()[b, 13]) == DISABLE_DEACTIVATION
