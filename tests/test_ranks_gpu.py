"""Two ranks on one GPU (each its own process and CUDA context; they wait for
each other only on the host, through the stand-in MPI's sockets), device
buffers: strided sends between the ranks by DEVICE, ONE_SHOT and STAGED;
the multi-rank periodic halo exchange through the interposed
MPI_Neighbor_alltoallw (edges to the other rank: TEMPI's Isend/Irecv
sequence with its own pack and unpack kernels) and through the reference's
MPI_Pack / MPI_Neighbor_alltoallv / MPI_Unpack sequence; and the interposed
MPI_Alltoallv by each of its methods.  Every rank checks its result against
the oracle."""
import pytest

from .ranks import run_ranks

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scenario", ["p2p", "halo", "alltoallv"])
def test_two_ranks_device(cuda, scenario):
    codes, outs = run_ranks(2, scenario, device=True, timeout=300)
    assert codes == [0, 0], "\n".join(o[-3000:] for o in outs)
    for r, o in enumerate(outs):
        assert f"rank {r} of 2: {scenario} ok" in o
