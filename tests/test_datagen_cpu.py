"""The package's inverse-CDF tables equal the oracle's, so device columns
drawn with them are the oracle's columns."""
import numpy as np
import pytest

from engine_b200 import datagen


@pytest.mark.parametrize("s,n", [(1.2, 1 << 20), (1.1, 1000), (1.5, 7), (0.8, 1)])
def test_zipf_table(orc, s, n):
    assert np.array_equal(datagen.zipf_table(s, n), orc.zipf_table(s, n))


@pytest.mark.parametrize("p", [0.25, 0.5, 1 / 32, 0.9])
def test_geom_table(orc, p):
    assert np.array_equal(datagen.geom_table(p), orc.geom_table(p))
