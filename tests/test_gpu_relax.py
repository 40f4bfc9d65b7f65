"""QuickMin relaxation on the CUDA engine against the oracle (GPU)."""
import pytest

from test_relax import check_quickmin_matches_oracle

pytestmark = pytest.mark.gpu


def test_quickmin_matches_oracle_on_gpu(gpu_engine):
    check_quickmin_matches_oracle(gpu_engine)


def test_cg2_matches_oracle_on_gpu(gpu_engine):
    from test_relax import check_cg2_matches_oracle
    check_cg2_matches_oracle(gpu_engine)


def test_bfgs_matches_oracle_on_gpu(gpu_engine):
    from test_relax import check_bfgs_matches_oracle
    check_bfgs_matches_oracle(gpu_engine)


def test_gradient_cg_matches_oracle_on_gpu(gpu_engine):
    from test_relax import check_gradient_cg_matches_oracle
    check_gradient_cg_matches_oracle(gpu_engine)


def test_bfgs_wgc_matches_oracle_on_gpu(gpu_engine):
    from test_relax import check_bfgs_wgc_matches_oracle
    check_bfgs_wgc_matches_oracle(gpu_engine)
