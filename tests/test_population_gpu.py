"""tg_crater_generate_device (the crater population drawn on the device, one thread per
generation cell) against tg_crater_generate (the host restatement, bit-exact with the reference's
GenerateCraters: tests/test_population.py): the same craters in the same order, counts, positions,
ages, ids and diameters bit for bit (the diameters' roots correctly rounded when the inversion's
power -1 / e is exactly -q / p, p a power of two: e = 2, the craters' slope, e = 1, 4, 0.8, ...; a
root within 0.1 ulp of a rounding midpoint sends its cell to the host); with any other exponent
the diameters within the last bits of the device's `pow`; and with
a wide tolerance, which sends most cells reaching PTRS's acceptance test to the host, the same
craters."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    # (seed, coefficient, dmin, dmax, margin radii, region): PTRS cells (the benchmark's density),
    # multiplication cells, candidate margins, a region off the origin
    (7, 200000 / (2048.5**2 * (1.0 - 500.0**-2)), 1.0, 500.0, 0.0, (0.0, 0.0, 2048.5, 2048.5)),
    (3, 0.01, 1.0, 100.0, 0.0, (-300.0, 150.0, 500.0, 900.0)),
    (11, 0.05, 0.5, 40.0, 3.0, (1.0e6, 2.0e3, 1.0e6 + 400.0, 2.0e3 + 300.0)),
]


def _pop(seed, coefficient, dmin, dmax, margin):
    from terraingen_b200.workloads import crater_population

    p = crater_population(seed, coefficient, dmin, dmax)
    p.margin_radii = margin
    return p


@pytest.mark.parametrize("case", range(len(CASES)))
def test_device_population_is_the_host_population(device, case):
    from terraingen_b200.workloads import generate_craters, generate_craters_device

    seed, c, dmin, dmax, margin, region = CASES[case]
    host = generate_craters(_pop(seed, c, dmin, dmax, margin), region)
    dev = generate_craters_device(device, _pop(seed, c, dmin, dmax, margin), region)
    assert len(host["x"]) > 100
    for k in ("x", "y", "age", "id", "diameter"):
        assert np.array_equal(dev[k], host[k]), k


@pytest.mark.parametrize("exponent", [1.0, 4.0, 0.8])
def test_device_diameters_are_the_hosts_for_dyadic_powers(device, exponent):
    from terraingen_b200.workloads import crater_population, generate_craters, \
        generate_craters_device

    region = (-200.0, 100.0, 600.0, 700.0)
    pop = lambda: crater_population(5, 0.02, 1.0, 60.0, exponent=exponent)  # noqa: E731
    host = generate_craters(pop(), region)
    dev = generate_craters_device(device, pop(), region)
    assert len(host["x"]) > 100
    for k in ("x", "y", "age", "id", "diameter"):
        assert np.array_equal(dev[k], host[k]), k


@pytest.mark.parametrize("exponent", [2.1, 3.0])
def test_other_exponents_diameters_within_last_bits(device, exponent):
    from terraingen_b200.workloads import crater_population, generate_craters, \
        generate_craters_device

    region = (-200.0, 100.0, 600.0, 700.0)
    pop = lambda: crater_population(5, 0.02, 1.0, 60.0, exponent=exponent)  # noqa: E731
    host = generate_craters(pop(), region)
    dev = generate_craters_device(device, pop(), region)
    for k in ("x", "y", "age", "id"):
        assert np.array_equal(dev[k], host[k]), k
    rel = np.abs(dev["diameter"] - host["diameter"]) / host["diameter"]
    assert rel.max() <= 1e-14, rel.max()


def test_wide_tolerance_draws_on_the_host(device):
    # A wide tolerance flags most cells that reach PTRS's acceptance test: the host draws them and
    # the device writes the rest around them, in order. Their diameters are then the host's bits.
    from terraingen_b200.workloads import generate_craters, generate_craters_device

    seed, c, dmin, dmax, margin, region = CASES[0]
    host = generate_craters(_pop(seed, c, dmin, dmax, margin), region)
    narrow = generate_craters_device(device, _pop(seed, c, dmin, dmax, margin), region)
    wide = generate_craters_device(device, _pop(seed, c, dmin, dmax, margin), region,
                                   tolerance=0.5)
    for k in ("x", "y", "age", "id", "diameter"):
        assert np.array_equal(wide[k], host[k]), k
        assert np.array_equal(narrow[k], host[k]), k
