"""Hosek-Wilkie state cook (dr_sky_cook) against the reference's cook."""
import os

import numpy as np
import pytest

from conftest import golden
from droplet_b200 import sky

from oracle import reference_src

DATASET = os.path.join(reference_src(), "ArHosekSkyModelData_RGB.h")


@pytest.fixture(scope="module")
def dataset():
    if not os.path.exists(DATASET):
        pytest.skip("Hosek-Wilkie dataset header not present")
    return sky.load_dataset(DATASET)


def test_cook_matches_reference_states(dataset):
    for st in golden("sky_states.json"):
        s = sky.cook(dataset, st["turbidity"], st["albedo"], st["elevation"])
        assert np.array_equal(s.configs, np.asarray(st["configs"])), st["note"]
        assert np.array_equal(s.radiances, np.asarray(st["radiances"])), st["note"]


def test_cook_matches_reference_live(dataset, ref):
    rng = np.random.default_rng(2)
    for _ in range(50):
        T, A, E = rng.uniform(1, 10), rng.uniform(0, 1), rng.uniform(0, np.pi / 2)
        s = sky.cook(dataset, T, A, E)
        c, r = ref.sky_state(T, A, E)
        assert np.array_equal(s.configs, c) and np.array_equal(s.radiances, r)


def test_solar_elevation_matches_reference(ref):
    from droplet_b200 import camera as cam

    for el in (5.0, 30.0, 45.0, 80.0):
        sd = cam.sun_direction(el, 30.0)
        assert abs(sky.solar_elevation(sd) - ref.solar_elevation(sd)) <= 2e-7


def test_cook_rejects_out_of_range(dataset):
    from droplet_b200 import _native as N

    with pytest.raises(N.DrError):
        sky.cook(dataset, 11.0, 0.3, 0.5)
