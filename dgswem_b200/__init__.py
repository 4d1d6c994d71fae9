"""dgswem_b200 -- B200 (sm_100a) implementation of DG-SWEM's explicit DG hydro
time step (DG_HYDRO_TIMESTEP), a drop-in behind the C-ABI in
include/dgswem_cuda.h.

    from dgswem_b200 import Deck, HydroStep
    deck = Deck("case_dir")            # fort.14/15/dg(/13) -> PREP_DG setup
    with HydroStep(deck) as hs:        # device-resident state on cuda:0
        for it in range(1, nt + 1):
            hs.timestep(it)
        eta, uu, vv, nodecode = hs.modal2nodal()
"""
from .hydro import Deck, DistributedPartition, HydroStep, PartitionedRun, run_case, write_fort63, write_hotstart  # noqa: F401
from .ensemble import Ensemble  # noqa: F401

__all__ = ["Deck", "DistributedPartition", "Ensemble", "HydroStep", "PartitionedRun", "run_case", "write_fort63",
           "write_hotstart"]
