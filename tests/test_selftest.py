"""Device self-checks of arithmetic that restates IEEE operations with other instructions."""

from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def test_projection_factor_equals_ieee_sqrt_and_reciprocal_everywhere(cuda):
    """The FGP projection's 1 / sqrt(x), from approximate hardware results refined with FMAs, equals
    RN(1 / RN(sqrt(x))) -- the reference's 1.0f / std::sqrt(x) -- for every float in [1, 2^126)."""
    from qoraholo_b200 import capi

    mismatches, first = capi.selftest_rcp_sqrt()
    assert mismatches == 0, f"{mismatches} mismatches, first at x bits {first:#010x}"
