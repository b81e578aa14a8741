"""Options the GPU path does not compute are refused before any device
work, instead of running with different physics (CPU only)."""
import pytest

from swinmd_b200 import engine, systems


def _pw():
    return systems.polarizable_water(nmol=8, kmax=3, seed=1)


@pytest.mark.parametrize("field", ["compute_wolf"])
def test_unsupported_options_refused(field):
    # (Wolf is built, but not together with the multipoles)
    s = _pw()
    setattr(s.config, field, True)
    with pytest.raises(NotImplementedError):
        engine.refuse_unsupported(s.config)


def test_default_options_accepted():
    engine.refuse_unsupported(_pw().config)


def test_ub_with_constraints_refused():
    s = _pw()
    s.config.compute_ub = True
    with pytest.raises(NotImplementedError):
        engine.refuse_unsupported(s.config)


@pytest.mark.parametrize("name", ["MCY", "BBV", "CO2"])
def test_unsupported_molecule_kinds_refused(name):
    s = _pw()
    s.mol_type_names = [(name, 3)]
    with pytest.raises(NotImplementedError):
        engine.refuse_unsupported_molecules(s)
    engine.refuse_unsupported_molecules(_pw())   # "WAT" is built
