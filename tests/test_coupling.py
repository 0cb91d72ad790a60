"""Dof-map validation of goss_b200.coupling (host logic, no GPU)."""
from __future__ import annotations

import numpy as np
import pytest

from goss_b200.coupling import check_dof_maps


def test_valid_maps_pass():
    check_dof_maps(10, {"a": (4, np.array([0, 2, 4, 6])), "b": (3, np.array([1, 3, 9]))})


@pytest.mark.parametrize("maps", [
    {"a": (3, np.array([0, 1]))},                           # wrong length
    {"a": (2, np.array([0, 10]))},                          # out of range
    {"a": (2, np.array([-1, 0]))},
    {"a": (2, np.array([3, 3]))},                           # two nodes, one dof
    {"a": (2, np.array([0, 1])), "b": (2, np.array([1, 2]))},  # overlap
    {"a": (2, np.array([0.0, 1.0]))},                       # not integers
    {"a": (2, np.array([[0, 1]]))},
])
def test_invalid_maps_raise(maps):
    with pytest.raises(ValueError):
        check_dof_maps(10, maps)
