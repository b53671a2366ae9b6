"""The FP32-storage form against the FP64 form on the precision workload (honeycomb
graphene, 4,194,304 sites, 5000 moments): DOS and VAC within 1e-6 of the FP64
result (largest per-energy deviation relative to the peak). Four VAC steps here; the
full 20-step report is `python -m gpuqt_b200.precision_report`."""
from __future__ import annotations

import json

import pytest

from gpuqt_b200 import precision_report

pytestmark = pytest.mark.gpu


def test_graphene4m_fp32_within_1e6():
    r = precision_report.report("graphene4m", vac_steps=4)
    print(json.dumps(r))
    assert r["sites"] == 4194304 and r["moments"] == 5000
    assert r["dos"]["energy_rel_peak_max"] <= 1e-6
    assert r["vac"]["energy_rel_peak_max"] <= 1e-6
