"""NVE molecular dynamics of replicas on the CUDA engine against the oracle (GPU)."""
import pytest

from test_md import check_nve_matches_oracle, check_nvt_matches_oracle

pytestmark = pytest.mark.gpu


def test_nve_matches_oracle_on_gpu(gpu_engine):
    check_nve_matches_oracle(gpu_engine)


def test_nvt_matches_oracle_on_gpu(gpu_engine):
    check_nvt_matches_oracle(gpu_engine)


def test_npt_matches_oracle_on_gpu(gpu_engine):
    from test_md import check_npt_matches_oracle
    check_npt_matches_oracle(gpu_engine)


def test_npt_wgc_matches_oracle_on_gpu(gpu_engine):
    from test_md import check_npt_matches_oracle
    check_npt_matches_oracle(gpu_engine, nsteps=2, wgc=True)
