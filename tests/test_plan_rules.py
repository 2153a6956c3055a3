"""The single-pair planning rules of libslcs.so on CPU (slcs_pair_plan_info_sms
touches no device): rows per lane by SM sub-partition balance, row bands for
tall pairs, column strips for short wide ones, and columns per step.  The GPU
tests check that slcs_comb_pair follows the same plan on the device."""
import pytest

import slcs

B200_SMS = 148


def plan(m, n, sms=B200_SMS, **cfg):
    return slcs.pair_plan_info(m, n, slcs.Config.make(**cfg) if cfg else None, sms=sms)


def test_tall_square_pair_bands():
    p = plan(1 << 20, 1 << 20)
    assert (p["algo"], p["tile_m"], p["strips"], p["bands"]) == (slcs.ALGO_STRIPS, 14, 1, 8)
    assert p["stripes"] == 2341 and p["cols_per_step"] == 8 and p["braid_cutoff"] == 256


def test_rows_per_lane_follow_sub_partitions():
    # 2341 stripes of 14 rows fill 592 sub-partitions 4 deep; on 132 SMs
    # (528 sub-partitions) 2048 stripes of 16 rows need 4 and 2341 need 5.
    assert plan(1 << 20, 1 << 20)["tile_m"] == 14
    assert plan(1 << 20, 1 << 20, sms=132)["tile_m"] == 16
    for sms in (1, 8, 100, 148, 160):
        assert plan(1 << 20, 1 << 20, sms=sms)["tile_m"] in (12, 14, 16)


def test_narrow_tall_pair_takes_many_bands():
    p = plan((1 << 19) + 77, 700)
    assert p["algo"] == slcs.ALGO_STRIPS and p["bands"] == 16 and p["strips"] == 1
    assert p["cols_per_step"] == 4  # 74-stripe chains against 700 columns


def test_mid_size_pairs_take_strips_and_bands():
    p = plan(131072, 131072)
    assert (p["algo"], p["tile_m"], p["warps"], p["strips"], p["bands"]) == (slcs.ALGO_STRIPS, 16, 4, 4, 4)
    assert p["cols_per_step"] == 4
    assert plan(40000, 200000)["bands"] == 1  # below 2^16 rows: strips only
    assert plan(70000, 300000)["bands"] == 2


def test_small_pairs_stay_one_wavefront():
    p = plan(4096, 4096)
    assert (p["algo"], p["tile_m"], p["warps"], p["strips"], p["bands"]) == (slcs.ALGO_WAVEFRONT, 8, 4, 1, 1)
    assert p["stripes"] == 16 and p["braid_cutoff"] == 0


def test_configuration_wins():
    p = plan(1 << 20, 1 << 20, algo=slcs.ALGO_WAVEFRONT, tile_m=14, warps=8)
    assert (p["algo"], p["bands"], p["strips"]) == (slcs.ALGO_WAVEFRONT, 1, 1)
    assert p["cols_per_step"] == 4  # one chain of 2341 stripes: 8 columns would be slower
    p = plan(20000, 10007, algo=slcs.ALGO_STRIPS, strips=1, bands=8, tile_m=16)
    assert (p["bands"], p["stripes"], p["cols_per_step"], p["braid_cutoff"]) == (8, 40, 8, 1024)
    p = plan(3000, 3000, algo=slcs.ALGO_STRIPS, strips=3, bands=100, tile_m=4)
    assert p["bands"] == 24  # at most one band per stripe


def test_empty_and_invalid():
    assert plan(0, 5)["algo"] == 0 and plan(7, 0)["stripes"] == 0
    with pytest.raises(RuntimeError):
        plan(100, 100, tile_m=7)
    with pytest.raises(RuntimeError):
        plan(100, 100, sms=0)
