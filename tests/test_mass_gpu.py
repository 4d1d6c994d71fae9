"""Water volume of a closed basin on the device (GPU).

The nonlinear equations from a Gaussian bump of elevation in the closed,
flat basin of test_oracle_p2_convergence.py (land all round, no friction,
no forcing): sum_e (ZE_1 + HB_1) * area stays constant over 400 SSP(3,3)
steps at p=1 and p=2.  The FP64 builds (strict, fast) hold it to round-off
(1e-13 relative; the measured drift is about 1e-16).  The mixed build at
p=1 rounds each element's right-hand side to FP32 before the FP64 SSP
combination, so an edge flux's contributions to its two sides cancel only
to FP32 precision relative to the flux (measured drift 1.6e-14; at p=2 its
sums are FP64): 1e-12 relative.
"""
import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep

import test_oracle_p2_convergence as sw

pytestmark = pytest.mark.gpu

TOL = {"strict": 1e-13, "fast": 1e-13, "mixed": 1e-12}


@pytest.mark.parametrize("build", sorted(TOL))
@pytest.mark.parametrize("p", [1, 2])
def test_closed_basin_volume_on_device(built, tmp_path, p, build):
    path = tmp_path / f"mass_p{p}"
    ze, hb, area = sw.bump_state(path, p)
    kw = {"mixed": True} if build == "mixed" else {"strict": build == "strict"}
    with HydroStep(Deck(path), **kw) as hs:
        assert hs.dofh == ze.shape[1]
        zero = np.zeros_like(ze)
        hs.set_state(ze, zero, zero, np.ones(hs.ne, np.int32))
        hs.run(1, sw.NSTEPS)
        hs.synchronize()
        z, qx, _, wd = hs.state()
    vol0, vol1 = sw.water_volume(ze, hb, area), sw.water_volume(z, hb, area)
    print(f"p={p} {build}: volume drift {(vol1 - vol0) / vol0:.2e} after {sw.NSTEPS} steps")
    assert np.abs(qx).max() > 1e-4  # the bump spread
    assert np.all(wd == 1)
    assert abs(vol1 - vol0) <= TOL[build] * vol0, (vol0, vol1)
