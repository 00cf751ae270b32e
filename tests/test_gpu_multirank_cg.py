"""Multi-rank drop-in on a GPU: two ranks (gloo for the host buffers), the
root gathers the blocks and solves on its GPU; every rank's block of the
solution must equal the single-process GPU solve of the global system BIT
FOR BIT (same launch shape, same association), in-domain halos included."""
import pytest

from conftest import pkg
from test_multirank_cg import check_against_single, run_ranks

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [(12, 24, 16), (30, 60, 40)])
def test_two_ranks_on_one_gpu_match_single_process(tmp_path, dims):
    eaf = pkg()

    def solve(s, phi):
        with eaf.CGSolver(s.nr, s.nth, s.nz) as cg:
            res, nit, _ = cg.solve(s.arrays(), phi, 5000, 1e-8)
        return res, nit

    run_ranks(2, dims, tmp_path, use_gpu=True)
    check_against_single(2, dims, tmp_path, solve)
