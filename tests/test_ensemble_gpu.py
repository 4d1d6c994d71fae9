"""Batched ensemble (GPU): one handle on the merged members advances them in
the same kernel launches, and each member's result is bit for bit the one
of a handle on that member alone -- the per-element arithmetic and its order
do not depend on what else shares the launch (no atomics; node stars keep
each member's element order)."""
import numpy as np
import pytest

from dgswem_b200 import Ensemble, HydroStep, decks
from dgswem_b200.ensemble import make_members

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", ["fast", "strict", "mixed"])
def test_ensemble_matches_members_alone(built, scratch, variant):
    specs = decks.ensemble_specs(7, seed=5, ne_min=400, ne_max=6000)
    ds, met = make_members(scratch / f"ens_{variant}", specs, nsteps=60)
    kw = {"strict": variant == "strict", "mixed": variant == "mixed"}
    with Ensemble(ds, **kw) as ens:
        ens.set_met(*met)
        launches0 = ens.hs.kernel_launches
        ens.run(1, 60)
        ens.synchronize()
        # one launch per kernel and stage for all members
        assert ens.hs.kernel_launches - launches0 == 60 * ens.nrk * 3
        got = ens.states()
        got_nodal = ens.modal2nodal()
    for i, d in enumerate(ds):
        with HydroStep(d, **kw) as hs:
            hs.set_met(met[0][i], met[1][i], met[2][i])
            hs.run(1, 60)
            want = hs.state()
            want_nodal = hs.modal2nodal()
        for a, b, name in zip(got[i], want, ("ZE", "QX", "QY", "WDFLG")):
            np.testing.assert_array_equal(a, b, err_msg=f"member {i} {name}")
        for a, b, name in zip(got_nodal[i], want_nodal, ("ETA2", "UU2", "VV2", "NODECODE")):
            np.testing.assert_array_equal(a, b, err_msg=f"member {i} {name}")
    # the members moved: tides of different amplitude, wind, wet/dry
    assert all(np.abs(g[0]).max() > 0 for g in got)
