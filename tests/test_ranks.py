"""Several ranks on the CPU (host buffers): the stand-in MPI's transport
between processes, and TEMPI's interposed calls passing host-memory work to
it -- point-to-point in a ring with tags, MPI_ANY_SOURCE and large crossing
messages; a periodic halo exchange over a graph communicator whose edges go
to other ranks (MPI_Neighbor_alltoallw and the reference's MPI_Pack /
MPI_Neighbor_alltoallv / MPI_Unpack sequence); MPI_Alltoallv with uneven
blocks.  Each rank checks its results against the oracle."""
import pytest

from .ranks import run_ranks


@pytest.mark.parametrize("scenario", ["p2p", "halo", "alltoallv"])
@pytest.mark.parametrize("size", [2, 3])
def test_ranks_host(scenario, size):
    codes, outs = run_ranks(size, scenario)
    assert codes == [0] * size, "\n".join(o[-3000:] for o in outs)
    for r, o in enumerate(outs):
        assert f"rank {r} of {size}: {scenario} ok" in o
