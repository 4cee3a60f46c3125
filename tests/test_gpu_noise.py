"""The "philox" noise mode: the noise segment generated on the GPU (Philox4x32-10
+ Box-Muller), through the C ABI."""
import numpy as np
import pytest

import cases
import philox_ref as P
from cubnm_b200 import core

pytestmark = pytest.mark.gpu


def _args(seed, precision="fp64", noise_out=True, N=4, nodes=20, dur=8):
    args = list(cases.synthetic_args("rWW", N=N, nodes=nodes, duration_s=dur, seed=2, sim_seed=seed,
                                     G=np.linspace(0.5, 2, N), bold_remove_s=2, window_size=2, window_step=1,
                                     precision=precision))
    args[7] = dict(args[7], noise="philox")
    args[10] = noise_out
    return args


def test_device_noise_matches_the_restatement():
    """The Philox words are integers and match exactly; the Box-Muller values
    differ only by the rounding of log / sin / cos between CUDA and numpy
    (numpy rounds 2 pi u before cos; the kernel uses sincospi), a few 1e-16 near 0."""
    out = core.run_simulations(*_args(11))
    ref = P.philox_normals(11, out["_noise"].size)
    np.testing.assert_allclose(out["_noise"], ref, rtol=1e-13, atol=1e-14)


def test_philox_runs_are_reproducible_and_seeded():
    a = core.run_simulations(*_args(5))
    b = core.run_simulations(*_args(5, noise_out=False))
    c = core.run_simulations(*_args(6, noise_out=False))
    np.testing.assert_array_equal(a["sim_bold"], b["sim_bold"])
    assert np.abs(a["sim_bold"] - c["sim_bold"]).max() > 0


def test_philox_noise_fp32_within_bounds():
    o64 = core.run_simulations(*_args(3, noise_out=False, N=16, nodes=68, dur=30))
    o32 = core.run_simulations(*_args(3, precision="fp32", noise_out=False, N=16, nodes=68, dur=30))
    assert np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"]).max() <= 2e-3


def test_philox_init_is_faster_than_host_generation():
    """init_time: the noise segment (100 nodes, 30-s segment, 6e7 values) from the
    host mt19937 vs Philox on the GPU, each with a fresh seed."""
    def init_time(seed, mode):
        args = list(cases.synthetic_args("rWW", N=2, nodes=100, duration_s=4, seed=2, sim_seed=seed,
                                         bold_remove_s=1, window_size=2, window_step=1))
        args[7] = dict(args[7], noise=mode)
        return core.run_simulations(*args)["init_time"]
    t_host = init_time(101, "mt19937")
    t_gpu = init_time(102, "philox")
    print(f"noise segment: host mt19937 {t_host:.3f} s, GPU philox {t_gpu:.3f} s")
    assert t_gpu < t_host
