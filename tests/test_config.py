"""`ParticleBeam` reads as the reference's (``config.py:133-166``): nested tuples of its
positions, velocities and currents, equal and hashed by value, whether its fields have been
read yet or not."""

from __future__ import annotations

import copy
import dataclasses
import pickle

import numpy as np
import pytest

from beamtracer_b200.config import ParticleBeam


def _beam(position, velocity, current):
    return ParticleBeam("H+", position, velocity, current, charge=1.0, mass=1.007276)


P = np.arange(6.0).reshape(2, 3)
V = 1e5 * (P + 1.0)
C = [1e-3, 2e-3]


def test_fields_are_nested_tuples_of_floats():
    beam = _beam(P, V, C)
    assert len(beam) == 2
    assert beam.position == ((0.0, 1.0, 2.0), (3.0, 4.0, 5.0))
    assert type(beam.velocity) is tuple and type(beam.velocity[1]) is tuple
    assert beam.current == (1e-3, 2e-3) and type(beam.current[0]) is float


def test_beams_made_from_arrays_and_from_tuples_agree():
    a = _beam(P, V, C)
    b = _beam(tuple(map(tuple, P.tolist())), V.tolist(), tuple(C))
    assert a == b and hash(a) == hash(b)
    assert repr(a) == repr(b)
    assert dataclasses.asdict(a) == dataclasses.asdict(b)


@pytest.mark.parametrize("copier", [lambda b: pickle.loads(pickle.dumps(b)), copy.deepcopy,
                                    lambda b: dataclasses.replace(b, charge=1.0)])
def test_copies_of_an_unread_beam_equal_it(copier):
    fresh = _beam(P, V, C)
    assert copier(fresh) == _beam(P, V, C)


def test_arrays_are_read_only_copies_of_the_input():
    position = P.copy()
    beam = _beam(position, V, C)
    position[0, 0] = 99.0
    p, v, c = beam.arrays()
    assert p[0, 0] == 0.0 and beam.position[0][0] == 0.0
    with pytest.raises(ValueError):
        p[0, 0] = 1.0
    np.testing.assert_array_equal(v, V)
    np.testing.assert_array_equal(c, C)


def test_row_counts_must_agree():
    with pytest.raises(ValueError, match="one row per trajectory"):
        _beam(P, V, [1e-3])
