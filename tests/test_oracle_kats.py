"""The CPU oracle against the reference's own known-answer tests.

This pins the oracle: every case restates a unit test of
pgarrett-scripps/sequoia-boost (file:line in the case's `ref`)."""
import json
import os

import pytest

from engines import OracleEngine
from kat_checks import check_case

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "reference_kats.json")) as fh:
    CASES = json.load(fh)["cases"]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_reference_kat(case, orc, sb):
    check_case(case, OracleEngine(orc), sb.TrainingParams)
