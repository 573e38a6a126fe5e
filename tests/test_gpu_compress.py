"""Darby compression modes ("nu_R_nu_S", src/soap_turbo_compress.f90:120-303)
through the CUDA descriptor and force VJP, against the oracle fed the same
index maps: the kernels take any compression map, so these check the maps'
use (many kept components, several outputs per component, weights 1/sqrt 2
and sqrt 2) rather than new kernel code."""
import numpy as np
import pytest

from soap_turbo_b200 import synthetic as syn
from test_gpu_edge import check, make_nl, random_sites

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["0_0", "0_1", "0_2", "1_0", "1_1", "1_2", "2_0", "2_1", "2_2"])
def test_darby_modes_small_basis(mode):
    hp = syn.Hyper(alpha_max=[4, 4, 4], l_max=4, basis="poly3gauss", compress_mode=mode)
    nl = make_nl(random_sites(np.random.default_rng(17), 24, 3), 3)
    check(hp, nl)


@pytest.mark.parametrize("mode", ["1_1", "2_2"])
def test_darby_modes_benchmark_basis(mode):
    """The 3-species alpha = 8, l_max = 8 basis: 2_2 keeps all 2700
    components, 1_1 compresses them to 216."""
    hp = syn.Hyper(alpha_max=[8, 8, 8], l_max=8, basis="poly3gauss", compress_mode=mode)
    nl = make_nl(random_sites(np.random.default_rng(23), 16, 3, lo=30, hi=80), 3)
    check(hp, nl)


@pytest.mark.parametrize("basis", ["poly3", "poly3operator"])
def test_darby_mode_other_bases(basis):
    hp = syn.Hyper(alpha_max=[4, 4, 4], l_max=4, basis=basis, compress_mode="1_2")
    nl = make_nl(random_sites(np.random.default_rng(29), 20, 3), 3)
    check(hp, nl)
