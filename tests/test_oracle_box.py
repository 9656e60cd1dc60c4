"""Pins the oracle's whole box/mixed step to the reference's known-answer tests (see box_cases.py)."""
import pytest

import box_cases as C

FAST = [C.case_grid_finds_every_pair, C.case_free_fall, C.case_stable_spin, C.case_tumble_keeps_momentum_and_energy,
        C.case_head_on, C.case_column, C.case_flat_rests_flat, C.case_slope_holds, C.case_slope_slides,
        C.case_ball_rests_on_box, C.case_sliding_ball_rolls, C.case_rolling_resistance, C.case_ball_into_box,
        C.case_show]


@pytest.mark.parametrize("case", FAST, ids=lambda c: c.__name__)
def test_oracle_box_case(case):
    case("oracle")


def test_oracle_mixed_pile_rests():
    C.case_mixed_pile_rests("oracle")


def test_oracle_pile_of_343_rests():
    C.case_pile("oracle", threads=True)
