"""extend_scalar (ordito/heat.py:2321) on the device against the oracle's exact restatement."""

from __future__ import annotations

import warnings

import numpy as np
import pytest

from oracle import heat_path as hp
from ordito_b200 import creation
from ordito_b200 import heat as gheat
from ordito_b200.mesh import Trimesh
from tests import meshes

pytestmark = pytest.mark.gpu

# The device diffuses by the settled CG: every entry settled to 1e-6 of itself, so the quotient
# of the two columns to about that.
EXTEND_TOL = 1e-5


def test_extend_scalar_between_the_poles(gpu) -> None:
    v, f = creation.icosphere(3)
    heights = v[:, 2]
    poles = np.array([np.argmax(heights), np.argmin(heights)], dtype=np.int32)
    values = np.array([1.0, -1.0])
    got = gheat.extend_scalar(v, f.reshape(-1), poles, values).numpy()
    assert f"{got[heights > 0.5].min():.2f}" == "1.00"
    assert f"{got[heights < -0.5].max():.2f}" == "-1.00"
    ref, _ = hp.extend_scalar(v, f, poles, values)
    assert np.max(np.abs(got - ref)) <= EXTEND_TOL * 2.0


@pytest.mark.parametrize("name", ["bumpy_sphere", "small_torus", "saddle_graded"])
def test_extend_scalar_matches_the_oracle(gpu, name: str) -> None:
    v, f = meshes.ALL[name]()
    rng = np.random.default_rng(4)
    sources = rng.choice(v.shape[0], size=5, replace=False).astype(np.int32)
    values = rng.normal(size=5)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", UserWarning)  # obtuse faces may overshoot (checked below)
        got = gheat.extend_scalar(Trimesh(v, f.reshape(-1)), sources, values).numpy()
    ref, _ = hp.extend_scalar(v, f, sources, values)
    scale = np.ptp(values)
    assert np.max(np.abs(got - ref)) <= EXTEND_TOL * scale
    assert np.allclose(got[sources], ref[sources], atol=EXTEND_TOL * scale)


def test_extend_scalar_warns_where_obtuse_faces_overshoot(gpu) -> None:
    # ordito/heat.py:161-166: on the irregular fixtures negative weights push the quotient past the
    # source values' range; the oracle measures the same excess.
    v, f = meshes.sphere_irregular()
    sources = np.array([0, 100, 200, 300], dtype=np.int32)
    values = np.array([0.0, 1.0, 2.0, 3.0])
    _, excess = hp.extend_scalar(v, f, sources, values)
    if excess > 1e-4 * 3.0:
        with pytest.warns(UserWarning, match="leaves the source values' range"):
            gheat.extend_scalar(v, f.reshape(-1), sources, values)
    else:
        with warnings.catch_warnings():
            warnings.simplefilter("error", UserWarning)
            gheat.extend_scalar(v, f.reshape(-1), sources, values)


def test_extend_scalar_arguments(gpu) -> None:
    v, f = creation.icosphere(2)
    with pytest.raises(ValueError):
        gheat.extend_scalar(v, f.reshape(-1), np.array([0, v.shape[0]], dtype=np.int32), np.array([1.0, 2.0]))
    with pytest.raises(ValueError):
        gheat.extend_scalar(v, f.reshape(-1), np.array([0, 1], dtype=np.int32), np.array([1.0]))
    empty = gheat.extend_scalar(v, f.reshape(-1), np.array([], dtype=np.int32), np.array([]))
    assert empty.numpy().shape == (v.shape[0],) and not empty.numpy().any()
    # A repeated source adds its values and its indicator: the quotient is their mean.
    got = gheat.extend_scalar(v, f.reshape(-1), np.array([3, 3], dtype=np.int32), np.array([1.0, 3.0])).numpy()
    reached = got != 0.0
    assert reached.sum() > v.shape[0] // 2
    assert np.allclose(got[reached], 2.0, rtol=0.0, atol=1e-12)
