"""The oracle pinned to the reference: every snapshot of the reference's
golden fort.63.true files (quarter_annular, wetdry, mass_conservation) is
reproduced to the 8 printed digits, and the wet/dry dry-node mask bit for bit."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden_dir
from oracle_lib import lib, read_fort63, run_case


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_oracle_reproduces_golden(built, tmp_path, case):
    lib().orc_set_threads(8)
    out = tmp_path / "fort.63"
    run_case(golden_dir(case), out)
    its, eta = read_fort63(out)
    exp = np.load(golden_dir(case) / "expected.npz")
    np.testing.assert_array_equal(its, exp["it"])
    dry_o, dry_e = np.abs(eta) > 90000, np.abs(exp["eta"]) > 90000
    np.testing.assert_array_equal(dry_o, dry_e)
    wet = ~dry_e
    # print precision of E16.8: half a unit in the 8th significant digit
    tol = 5e-9 * np.maximum(1.0, 10.0 ** np.ceil(np.log10(np.maximum(np.abs(exp["eta"]), 1e-30))))
    assert (np.abs(eta - exp["eta"])[wet] <= tol[wet] + 1e-15).all()
