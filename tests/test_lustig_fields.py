"""CPU checks of the Lustig fixtures and the host-side Lustig virial: the
reference's LFIntegrator forms molVirt from the myLustig fields its force
terms wrote (src/integrators/LFIntegrator.cpp:731-734); engine.lustig_molvirt
must give the same number from the same fields, and the fixtures' field
order must be the one the library returns (SMD_LUS_*)."""
import numpy as np
import pytest

from conftest import golden
from swinmd_b200 import engine
from swinmd_b200 import _lib as L

CASES = ["nacl1000_lustig", "spcf216_lustig", "spce512_lustig", "spce512_wolf_lustig",
         "polwater216_lustig", "ref_test_lustig"]


@pytest.mark.parametrize("name", CASES)
def test_molvirt_from_fields(name):
    g = golden(name)
    fields = g["r_step_lustig_all"].reshape(-1, len(L.LUSTIG_FIELDS))
    vol = float(np.prod(g["box"]))
    for step in range(fields.shape[0]):
        f = dict(zip(L.LUSTIG_FIELDS, fields[step]))
        mv = engine.lustig_molvirt(f, vol)
        ref = g["r_step_molvirt"][step]
        assert abs(mv - ref) <= 1e-12 * max(1.0, abs(ref)), (step, mv, ref)


def test_field_order_matches_header():
    # the names in the ABI's order, against the header's enum
    import os
    import re
    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "swinmd_b200.h")).read()
    start = hdr.index("SMD_LUS_LJ_U = 0")
    body = hdr[start:hdr.index("SMD_LUSTIG_COUNT", start)]
    names = re.findall(r"SMD_LUS_\w+", body)
    assert len(names) == len(L.LUSTIG_FIELDS) == 29
