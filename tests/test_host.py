"""Host-side mirror of the reference interface (CPU only)."""
from pathlib import Path

import numpy as np

from cfd_inwsl_b200 import zone

GOLD = Path(__file__).resolve().parent / "golden"


def test_enums_match_reference_values():
    # macro.hpp:33-90
    assert zone.BndType.SUPERSONICOUTLET == 7 and zone.BndType.SYMMETRYY == 11
    assert zone.InterMethod.WCNS5 == 2 and zone.InterMethod.TCNS5 == 11 and zone.InterMethod.INTERMAX == 16
    assert zone.InterMethod.new_TCNS5 == 35 and zone.InterMethod.new_WHFTCNSASF202_NoS == 39
    assert zone.FluxMethod.HLLC == 0 and zone.FluxMethod.ROE == 1
    assert zone.DiffMethod.MND6 == 3


def test_info_defaults_and_grid():
    info = zone.Info()
    assert info.dim == 2 and info.icMax() == [200, 200, 1]
    assert info.fluxMethod == zone.FluxMethod.ROE and info.CFL == 0.5
    info.iMax = [401, 1, 1]
    info.calZone = [-0.5, 0.5, 0, 0, 0, 0]
    assert info.icMax() == [400, 1, 1]
    assert info.geth(0) == (0.5 - -0.5) / 400 and info.geth(1) == info.geth(0)
    assert info.nGhostCell() == 4
    info.diffMethod = zone.DiffMethod.TRAD6
    assert info.nGhostCell() == 5  # info.cpp:10


def test_default_bc_types_follow_initializer():
    info = zone.Info()
    info.dim = 2
    for ncase, exp in [(0, [7, 7]), (2, [10, 11]), (3, [10, 3]), (6, [1, 1])]:
        info.nCase = ncase
        bc = zone.default_bc_types(info)
        assert [bc[0][0], bc[1][0]] == exp
    info.dim = 1
    info.nCase = 4
    assert zone.default_bc_types(info)[0] == [zone.BndType.SYMMETRY1D] * 2


def test_sod_initial_state_matches_reference():
    info = zone.Info()
    info.iMax = [401, 1, 1]
    info.calZone = [-0.5, 0.5, 0, 0, 0, 0]
    info.dim = 1
    g = np.load(GOLD / "sod_400.npz")
    np.testing.assert_array_equal(zone.sod_1d(info), g["cons0"])
