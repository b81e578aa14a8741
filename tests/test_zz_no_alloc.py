"""The force entry point that allocates no device memory gives exactly the
results of smd_compute_forces, on two calls in a row, and refuses systems
larger than its static scratch."""
import numpy as np
import pytest

from swinmd_b200 import engine, systems
from swinmd_b200 import _lib as L

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_matches_compute_forces(precision):
    s = systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3, n_steps=10)
    ens = engine.GpuEnsemble(s, precision=precision)
    f0, e0, w0 = ens.compute_forces()
    for _ in range(2):
        f1, e1, w1 = ens.compute_forces_noalloc()
        assert np.array_equal(f0, f1)
        assert np.array_equal(e0, e1)
        assert np.array_equal(w0, w1)
    ens.close()


def test_noalloc_rejects_oversize():
    s = systems.lj_fluid(ncell=26, seed=1)   # 70304 atoms > 65536
    ens = engine.GpuEnsemble(s)
    with pytest.raises(L.SmdError) as ex:
        ens.compute_forces_noalloc()
    assert "65536" in str(ex.value)
    ens.close()
