"""The host functions both arms share, against the reference's own outputs.

The beam seeding, the plane moments and the axisymmetric magnetic field of this package
feed the device path and the oracle alike, so the oracle cannot check them: the fixtures
``tests/golden/host_*.npz`` were made by running the reference's ``beam_with_energy``
(``solver/tracer.py:221-291``), ``plane_moments`` (``solver/diagnostics.py:56-135``),
``AxisymmetricMagneticField`` and ``solenoid_on_axis`` (``solver/fields.py:192-321``) and
its solenoid sampling (``model.py:169-188``) on the cases of ``tests/golden/host_cases.py``.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from beamtracer_b200.diagnostics import BeamMoments, mismatch, plane_moments
from beamtracer_b200.fields import AxisymmetricMagneticField, solenoid_on_axis
from beamtracer_b200.model import config_magnetic_field
from beamtracer_b200.tracer import PlaneHits, beam_with_energy
from tests.golden import host_cases as hc
from tests.gpu_util import GOLDEN

RTOL = 1e-12


@pytest.fixture(scope="module")
def beams():
    return np.load(GOLDEN / "host_beams.npz")


@pytest.mark.parametrize("name", sorted(hc.BEAM_CASES))
def test_beam_matches_the_reference(beams, name):
    args, kwargs = hc.BEAM_CASES[name]
    kwargs = dict(kwargs)
    if "seed" in kwargs:
        kwargs["sampling"] = np.random.default_rng(kwargs.pop("seed"))
    particles, j_over_v = beam_with_energy(*args, **kwargs)
    for key in ("position", "velocity", "charge", "mass", "current"):
        want = beams[f"{name}.{key}"]
        got = getattr(particles, key)
        assert got.shape == want.shape, key
        np.testing.assert_allclose(got, want, rtol=RTOL, atol=RTOL * np.abs(want).max(),
                                   err_msg=key)  # fmt: skip
    np.testing.assert_array_equal(particles.species, beams[f"{name}.species"])
    assert j_over_v == pytest.approx(float(beams[f"{name}.j_over_v"]), rel=RTOL)


def _hits(name: str) -> tuple[PlaneHits, dict]:
    seed, cylindrical, species, forward, axis, mass_kind = hc.MOMENT_CASES[name]
    h = hc.moment_hits(seed, cylindrical)
    if name == "planar_fast":
        h["velocity"] = h["velocity"] * 150.0
    hits = PlaneHits(0.0)
    hits.append(h["point"], h["velocity"], h["current"], h["species"], h["direction"])
    mass = hc.MOMENT_MASSES if mass_kind == "array" else float(hc.MOMENT_MASSES[0])
    return hits, {"cylindrical": cylindrical, "mass": mass, "species": species,
                  "forward_only": forward, "axis": axis}  # fmt: skip


@pytest.mark.parametrize("name", sorted(hc.MOMENT_CASES))
def test_moments_match_the_reference(name):
    golden = np.load(GOLDEN / "host_moments.npz")[name]
    hits, kwargs = _hits(name)
    m = plane_moments(hits, **kwargs)
    got = np.array([getattr(m, k) for k in BeamMoments.__dataclass_fields__], dtype=float)
    np.testing.assert_allclose(got, golden, rtol=RTOL, atol=0.0)


def test_ring_moments_are_those_of_the_rotated_rings():
    """The reference's known answer (``tests/unit/test_ion_optics.py:258-281``): a ring's
    moments equal those of its points spread over the azimuth."""
    rng = np.random.default_rng(1)
    n = 300
    r = rng.uniform(0, 3e-3, n)
    rp = 5.0 * r + rng.normal(0, 1e-3, n)
    ap = rng.normal(0, 2e-3, n)
    w = rng.uniform(0.5, 1.5, n)
    hits = PlaneHits(0.0)
    hits.append(np.stack([np.zeros(n), r, np.zeros(n)]), np.stack([np.ones(n), rp, ap]), w,
                np.zeros(n, dtype=np.int32), np.ones(n, dtype=np.int8))  # fmt: skip
    ring = plane_moments(hits, cylindrical=True, mass=1.0)
    theta = np.linspace(0, 2 * np.pi, 720, endpoint=False)
    x = (r[:, None] * np.cos(theta)).ravel()
    xp = (rp[:, None] * np.cos(theta) - ap[:, None] * np.sin(theta)).ravel()
    ww = np.repeat(w, theta.size)
    xx, pp, xpp = (np.average(q, weights=ww) for q in (x * x, xp * xp, x * xp))
    assert ring.emittance == pytest.approx(np.sqrt(xx * pp - xpp**2), rel=1e-9)
    assert ring.alpha == pytest.approx(-xpp / ring.emittance, rel=1e-9)


def test_no_forward_crossings_give_nan_moments():
    hits = PlaneHits(0.0)
    hits.append(np.zeros((3, 2)), np.ones((3, 2)), np.ones(2), np.zeros(2, np.int32),
                -np.ones(2, np.int8))  # fmt: skip
    m = plane_moments(hits, cylindrical=True, mass=1.0)
    assert m.current == 0.0 and m.count == 0 and np.isnan(m.emittance)


def test_matched_beam_has_no_mismatch():
    """The reference's known answers for the mismatch (``test_ion_optics.py:284-286``)."""
    assert mismatch(1.02, 0.11, 1.02, 0.11) == pytest.approx(0.0, abs=1e-12)
    assert mismatch(0.0, 0.2, 1.02, 0.11) > 0.1


@pytest.mark.parametrize("name", sorted(hc.FIELD_CASES))
def test_magnetic_field_matches_the_reference(name):
    golden = np.load(GOLDEN / "host_fields.npz")
    centre, length, radius, peak, z0, hz, n, order = hc.FIELD_CASES[name]
    profile = solenoid_on_axis(z0 + hz * np.arange(n), centre, length, radius, peak)
    np.testing.assert_allclose(profile, golden[f"{name}.profile"], rtol=0,
                               atol=RTOL * abs(peak))  # fmt: skip
    field = AxisymmetricMagneticField(z0, hz, golden[f"{name}.profile"], order=order)
    table = golden[f"{name}.table"]
    from beamtracer_b200.fields import _derivative_weights

    weights = np.abs(_derivative_weights()).sum(axis=1)
    for k in range(order + 1):  # each derivative to the rounding bound of its stencil
        bound = 8 * np.finfo(float).eps * weights[k] * np.abs(profile).max() / hz**k
        np.testing.assert_allclose(field.samples[:, k], table[:, k], rtol=0, atol=bound,
                                   err_msg=f"d^{k}")  # fmt: skip
    # The k-th difference stencil cancels to hz^k B^(k) from terms of size B: its rounding
    # is amplified by ~ sum|c| / (hz^k |B^(k)|), and a sum of the seven terms in another
    # order moves B_r's r^3 B^(3) term by ~1e-11 T here.  1e-10 of the peak bounds that.
    z, r = hc.field_points(30 + list(hc.FIELD_CASES).index(name), z0, hz, n)
    bz, br = field(z, r)
    np.testing.assert_allclose(bz, golden[f"{name}.bz"], rtol=0, atol=1e-10 * abs(peak))
    np.testing.assert_allclose(br, golden[f"{name}.br"], rtol=0, atol=1e-10 * abs(peak))


def test_solenoid_sampling_matches_the_reference():
    """A configuration's solenoids sampled every half node spacing over the mesh and eight
    samples beyond each end, as ``BeamOptics`` does (``model.py:169-188``)."""
    golden = np.load(GOLDEN / "host_fields.npz")
    lo, hi, h, solenoids, order = hc.SAMPLING_CASE
    config = SimpleNamespace(
        solenoids=[SimpleNamespace(centre=c, length=length, radius=a, peak=b)
                   for c, length, a, b in solenoids],
        axial_field=None, field_order=order)  # fmt: skip
    mesh = SimpleNamespace(h=h, origin=(lo, 0.0), upper=(hi, 1e-3))
    field = config_magnetic_field(config, mesh)
    assert field.bz.size == int(golden["sampling.count"])
    assert field.z0 == pytest.approx(float(golden["sampling.z0"]), abs=1e-18)
    z, r = hc.field_points(40, lo, h, int((hi - lo) / h))
    bz, br = field(z, r)
    peak = max(abs(b) for *_, b in solenoids)  # the stencils' rounding, as above
    np.testing.assert_allclose(bz, golden["sampling.bz"], rtol=0, atol=1e-10 * peak)
    np.testing.assert_allclose(br, golden["sampling.br"], rtol=0, atol=1e-10 * peak)
