"""Pins the CPU oracle's islands and sleeping against the reference's own island tests.

Each test restates the assertions of one test of crates/bullet-dynamics/src/world/islands.rs
(the `tests` module from line 309; each test's lines are cited), in both precisions.
"""
import numpy as np
import pytest

from oracle_api import (ACTIVE, DISABLE_DEACTIVATION, DISABLE_SIMULATION, ISLAND_SLEEPING, JOINT_POINT2POINT,
                        NO_CONTACT_RESPONSE, WANTS_DEACTIVATION, OracleWorld, frame, joint_desc)

PRECISIONS = ["f32", "f64"]
DT = 1.0 / 60.0
DEFAULT, ALL = 1, 0xFFFF  # body.rs:160-170 filter groups


def act(w, i):
    return int(w.state()[i, 13])


def is_active(w, i):
    # body.rs:524-532
    return act(w, i) in (ACTIVE, WANTS_DEACTIVATION, DISABLE_DEACTIVATION)


def run(w, steps, before=None):
    for _ in range(steps):
        if before:
            before()
        w.step(DT)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_body_sleeps_after_resting(prec):
    # world/islands.rs:317-346: after 3 s the resting sphere sleeps with zero velocity, and
    # further steps leave it where it is.
    w = OracleWorld(prec)
    w.add_body(w.plane([0, 1, 0], 0.0), [0, 0, 0], mass=0)
    s = w.add_body(w.sphere(0.5), [0, 2, 0], mass=1.0)
    run(w, int(3.0 / DT))
    st = w.state()[s]
    assert int(st[13]) == ISLAND_SLEEPING
    assert tuple(st[7:10]) == (0.0, 0.0, 0.0)
    y = st[1]
    run(w, 60)
    assert w.state()[s, 1] == pytest.approx(y, abs=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_contact_wakes_sleeping_body(prec):
    # world/islands.rs:353-393: a sphere asleep on the plane is woken by a ball dropped on it.
    w = OracleWorld(prec)
    w.add_body(w.plane([0, 1, 0], 0.0), [0, 0, 0], mass=0)
    s = w.add_body(w.sphere(0.5), [0, 1, 0], mass=1.0)
    run(w, int(3.0 / DT))
    assert act(w, s) == ISLAND_SLEEPING
    w.add_body(w.sphere(0.25), [0, 3, 0], linvel=(0, -5, 0), mass=1.0)
    run(w, 60)
    assert is_active(w, s)
    assert act(w, s) != ISLAND_SLEEPING


@pytest.mark.parametrize("prec", PRECISIONS)
def test_force_wakes_sleeping_body(prec):
    # world/islands.rs:397-417: applying a force makes a sleeping body Active at once.
    w = OracleWorld(prec)
    w.add_body(w.plane([0, 1, 0], 0.0), [0, 0, 0], mass=0)
    s = w.add_body(w.sphere(0.5), [0, 1, 0], mass=1.0)
    run(w, int(3.0 / DT))
    assert act(w, s) == ISLAND_SLEEPING
    w.apply_force(s, (0, 5, 0))
    assert act(w, s) == ACTIVE


@pytest.mark.parametrize("prec", PRECISIONS)
def test_static_body_starts_sleeping(prec):
    # world/islands.rs:423-430
    w = OracleWorld(prec)
    b = w.add_body(w.sphere(0.5), [0, 0, 0], mass=0)
    assert act(w, b) == ISLAND_SLEEPING
    assert not is_active(w, b)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_island_sleeps_and_wakes_as_unit(prec):
    # world/islands.rs:436-499: two touching boxes sleep together, stay frozen, and both wake
    # when a fast ball joins their island.
    w = OracleWorld(prec)
    w.set_gravity((0, -9.81, 0))
    w.add_body(w.plane([0, 1, 0], 0.0), [0, 0, 0], mass=0)
    cube = w.box([0.5, 0.5, 0.5])
    a = w.add_body(cube, [-0.5, 0.5, 0], mass=1.0)
    b = w.add_body(cube, [0.5, 0.5, 0], mass=1.0)
    run(w, int(4.0 / DT))
    assert not is_active(w, a) and not is_active(w, b)
    pa, pb = w.state()[a, 0:3].copy(), w.state()[b, 0:3].copy()
    run(w, 60)
    assert np.linalg.norm(w.state()[a, 0:3] - pa) < 1e-9
    assert np.linalg.norm(w.state()[b, 0:3] - pb) < 1e-9
    w.add_body(w.sphere(0.25), [-3.0, 0.5, 0.0], linvel=(8, 0, 0), mass=1.0)
    run(w, 30)
    assert is_active(w, a) and is_active(w, b)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_disable_deactivation_keeps_island_awake(prec):
    # world/islands.rs:508-536: a box stacked on a DisableDeactivation box never sleeps.
    w = OracleWorld(prec)
    w.set_gravity((0, -9.81, 0))
    w.add_body(w.plane([0, 1, 0], 0.0), [0, 0, 0], mass=0)
    cube = w.box([0.5, 0.5, 0.5])
    lo = w.add_body(cube, [0, 0.5, 0], mass=1.0, activation=DISABLE_DEACTIVATION)
    hi = w.add_body(cube, [0, 1.5, 0], mass=1.0)
    run(w, int(10.0 / DT))
    assert is_active(w, lo) and is_active(w, hi)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_joint_links_islands_across_a_distance(prec):
    # world/islands.rs:543-572: a point-to-point joint keeps a still, distant partner of a
    # driven body awake.
    w = OracleWorld(prec)
    w.set_gravity((0, 0, 0))
    ball = w.sphere(0.5)
    a = w.add_body(ball, [4.0, 0, 0], mass=1.0)
    b = w.add_body(ball, [6.0, 0, 0], mass=1.0)
    w.add_joint(joint_desc(JOINT_POINT2POINT, a, b, frame([1, 0, 0]), frame([-1, 0, 0]), flags=0))
    run(w, int(6.0 / DT), before=lambda: w.apply_force(a, (2, 0, 0)))
    assert is_active(w, b)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_moving_kinematic_wakes_sleeping_island(prec):
    # world/islands.rs:578-611: a kinematic slab flying in wakes the box asleep in its path.
    w = OracleWorld(prec)
    w.set_gravity((0, -10, 0))
    w.add_body(w.plane([0, 1, 0], 0.0), [0, 0, 0], mass=0)
    bx = w.add_body(w.box([0.25, 0.25, 0.25]), [0, 0.25, 0], mass=1.0)
    run(w, 600)
    assert not is_active(w, bx)
    w.add_body(w.box([0.5, 0.5, 0.5]), [-4.0, 0.25, 0.0], linvel=(6, 0, 0), mass=0, kinematic=1)
    woke = False
    for _ in range(120):
        w.step(DT)
        if is_active(w, bx):
            woke = True
            break
    assert woke


@pytest.mark.parametrize("prec", PRECISIONS)
def test_group_mask_excluded_pair_does_not_pin_island_awake(prec):
    # world/islands.rs:620-666: an always-awake body overlapping a still one through a pair the
    # group / mask test excludes leaves it to sleep; once the pair is made eligible it pins the
    # still body awake.
    w = OracleWorld(prec)
    w.set_gravity((0, 0, 0))
    ball = w.sphere(0.5)
    b = w.add_body(ball, [0, 0.5, 0], mass=1.0, group=2, mask=3)
    a = w.add_body(ball, [0.72, 0.5, 0.72], mass=1.0, group=DEFAULT, mask=DEFAULT, activation=DISABLE_DEACTIVATION)
    run(w, int(3.5 / DT))
    assert act(w, b) == ISLAND_SLEEPING
    w.set_filter(a, DEFAULT, ALL)
    run(w, 60)
    assert act(w, b) != ISLAND_SLEEPING


@pytest.mark.parametrize("prec", PRECISIONS)
@pytest.mark.parametrize("sensor", [False, True])
def test_sensor_body_does_not_pin_island_awake(prec, sensor):
    # world/islands.rs:674-710: an awake plain body pins its overlapping neighbour awake; an
    # awake sensor (NO_CONTACT_RESPONSE) does not merge islands and lets it sleep.
    w = OracleWorld(prec)
    w.set_gravity((0, 0, 0))
    ball = w.sphere(0.5)
    b = w.add_body(ball, [0, 0.5, 0], mass=1.0)
    w.add_body(ball, [0.72, 0.5, 0.72], mass=1.0, activation=DISABLE_DEACTIVATION,
               flags=NO_CONTACT_RESPONSE if sensor else 0)
    run(w, int(3.5 / DT))
    if sensor:
        assert act(w, b) == ISLAND_SLEEPING
    else:
        assert act(w, b) != ISLAND_SLEEPING


@pytest.mark.parametrize("prec", PRECISIONS)
def test_moving_kinematic_does_not_wake_group_excluded_body(prec):
    # world/islands.rs:716-753: a moving kinematic does not wake a sleeping box whose pair with it
    # the group / mask test excludes.
    w = OracleWorld(prec)
    w.set_gravity((0, -10, 0))
    w.add_body(w.plane([0, 1, 0], 0.0), [0, 0, 0], mass=0)
    bx = w.add_body(w.box([0.25, 0.25, 0.25]), [0, 0.25, 0], mass=1.0, group=2, mask=3)
    run(w, 600)
    assert not is_active(w, bx)
    w.add_body(w.box([0.5, 0.5, 0.5]), [-4.0, 0.25, 0.0], linvel=(6, 0, 0), mass=0, kinematic=1, group=DEFAULT,
               mask=DEFAULT)
    run(w, 120)
    assert not is_active(w, bx)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_disable_simulation_body_bridges_islands(prec):
    # world/islands.rs:761-816: a DisableSimulation body merges islands without being an awake
    # contributor and without its own state ever being rewritten: the still body beside it
    # sleeps, then wakes through it once an awake body joins on the other side.
    w = OracleWorld(prec)
    w.set_gravity((0, 0, 0))
    ball = w.sphere(0.5)
    b = w.add_body(ball, [1.02, 0, 0], mass=1.0, activation=DISABLE_SIMULATION)
    c = w.add_body(ball, [2.04, 0, 0], mass=1.0)
    run(w, int(3.5 / DT))
    assert act(w, c) == ISLAND_SLEEPING
    assert act(w, b) == DISABLE_SIMULATION
    w.add_body(ball, [0, 0, 0], mass=1.0, activation=DISABLE_DEACTIVATION)
    run(w, 30)
    assert is_active(w, c)
    assert act(w, b) == DISABLE_SIMULATION
