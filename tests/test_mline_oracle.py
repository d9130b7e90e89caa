"""The moving-line oracle (oracle/oracle_mline.c, FiniteVolume<1> with Motion::moving) against the reference's own moving
1D checks (src/test/hydro1d_test.cpp:121-514, restated in tests/mline_checks.py), on the CPU: no reference-held numbers
exist for the moving line, so these properties pin the restatement."""
import pytest

import mline_checks as C
from oracle import oracle as O

make = O.OracleMovingLine


@pytest.mark.parametrize("order", [0, 1])
def test_uniform_states_stay_uniform(order):
    C.uniform_states_stay_uniform(make, order)


@pytest.mark.parametrize("periodic", [True, False])
def test_conservation_and_same_bits(periodic):
    C.conservation_and_same_bits(make, periodic)


@pytest.mark.parametrize("n,bounds", [(128, (0.0063, 0.0097, 0.0047)), (256, (0.0034, 0.0046, 0.0023))])
@pytest.mark.parametrize("jitter", [0.0, 0.5])
def test_sod_within_luna_bounds(n, bounds, jitter):
    C.sod_within_luna_bounds(make, n, bounds, jitter)


def test_a_split_at_each_wall():
    C.a_split_at_each_wall(make)


@pytest.mark.parametrize("from_left", [True, False])
def test_supersonic_inflow_makes_a_lattice(from_left):
    C.supersonic_inflow_makes_a_lattice(make, from_left)


def test_shu_osher_budget_cells_and_mirror():
    C.shu_osher_budget_cells_and_mirror(make)


def test_fused_step_conserves_and_is_close():
    C.fused_step_conserves_and_is_close(make)


@pytest.mark.parametrize("name", ["sod", "woodward-colella"])
def test_no_cells_where_no_gas_enters(name):
    C.no_cells_where_no_gas_enters(make, name)
