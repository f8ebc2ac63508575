"""Size-independent properties at the configurations' full sizes (the oracle
cannot run 1024^2 / 2048^2 fields in seconds; the parity tests pin smaller
ones):

* conservation: the finite-volume flux form conserves mass, both momenta
  and total energy exactly in a periodic box without gravity (the face
  fluxes telescope), so the domain sums change only by FP64 round-off of
  the sums and updates -- for the FP64 and the mixed-precision path;
* mirror symmetry: a centred bubble at rest in a periodic box stays
  symmetric under x -> -x and y -> -y (with the odd momentum component
  changing sign), to FP64 round-off.
"""
import numpy as np
import pytest

from tests.helpers import interior

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    from dim2d_finite_volume_b200 import field
    return field


def _run(F, n, precision, steps, variant=2, radius=0.1):
    from dim2d_finite_volume_b200 import workloads
    d = workloads.domain(n, T0=0.95, bubbles=[(0.0, 0.0, radius)], bc="periodic_xy")
    with F.Field(d["nx"], d["ny"], bc="periodic_xy", precision=precision) as fld:
        fld.variant = variant
        fld.ini(d["nodes"], d["x_map"], d["y_map"])
        fld.integrate(d["dt"], steps)
        return d["nodes"], fld.download()


@pytest.mark.parametrize("n,precision", [(1024, 0), (1024, 1), (2048, 0)])
def test_conservation_periodic(F, n, precision):
    q0, q1 = _run(F, n, precision, 20)
    assert np.isfinite(q1).all()
    a, b = interior(q0), interior(q1)
    for k in range(4):
        scale = np.abs(a[k]).sum()
        drift = abs(b[k].sum() - a[k].sum())
        # the momenta start at 0: measure their drift against the mass
        ref = scale if scale > 0 else np.abs(a[0]).sum()
        assert drift <= 1e-12 * ref, (k, drift / ref)


@pytest.mark.parametrize("precision", [0, 1])
def test_mirror_symmetry_1024(F, precision):
    _, q = _run(F, 1024, precision, 20)
    c = interior(q)
    scale = np.abs(c).reshape(4, -1).max(axis=1)
    mx = c[:, :, ::-1].copy()   # x -> -x
    mx[1] *= -1.0
    my = c[:, ::-1, :].copy()   # y -> -y
    my[2] *= -1.0
    tol = 1e-12 if precision == 0 else 1e-6
    for k in range(4):
        assert np.abs(mx[k] - c[k]).max() <= tol * scale[k] + 1e-300, ("x", k)
        assert np.abs(my[k] - c[k]).max() <= tol * scale[k] + 1e-300, ("y", k)
