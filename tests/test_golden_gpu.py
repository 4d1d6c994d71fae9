"""The reference's golden tests, run on the CUDA path (GPU).

Mirrors the reference's tests/test_run.py: run each case to completion,
compare the last snapshot of nodal elevation (fort.63) with fort.63.true using
the reference's own tolerances (tests/test_run.py:8-24), and additionally
every snapshot against the printed values at print precision plus the
dry-node mask bit for bit.
"""
import numpy as np
import pytest

from conftest import golden_dir
from dgswem_b200 import run_case

pytestmark = pytest.mark.gpu

# (case, rtol, atol) exactly as tests/test_run.py of the reference
CASES = [("quarter_annular", 0.05, 1e-7), ("wetdry", 0.01, 1e-7), ("mass_conservation", 1e-3, 1e-7)]


@pytest.mark.parametrize("case,rtol,atol", CASES)
def test_golden(built, tmp_path, case, rtol, atol):
    snaps = run_case(golden_dir(case), out=tmp_path / "fort.63")
    exp = np.load(golden_dir(case) / "expected.npz")
    its = np.array([it for it, _ in snaps])
    got = np.array([eta for _, eta in snaps])
    np.testing.assert_array_equal(its, exp["it"])
    # the reference's assertion (last snapshot)
    np.testing.assert_allclose(got[-1], exp["eta"][-1], rtol=rtol, atol=atol)
    # stronger: every snapshot at the 8-digit print precision, same dry nodes
    dry_g, dry_e = np.abs(got) > 90000, np.abs(exp["eta"]) > 90000
    np.testing.assert_array_equal(dry_g, dry_e)
    wet = ~dry_e
    scale = np.maximum(np.abs(exp["eta"]), 1e-30)
    assert (np.abs(got - exp["eta"])[wet] <= 1e-8 * scale[wet] + 5e-9).all()
