"""The FP32 engine against the same engine tracking and sampling in FP64
(FP64 tables, IEEE arithmetic; same seed, same random draws): every
tally's difference must vanish next to its own Monte Carlo noise."""
import pytest

from chatcarlo_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_fp32_tracking_error_is_far_below_the_statistical_error():
    from chatcarlo_b200.precision import tally_precision
    from chatcarlo_b200.transport import Engine, default_engine
    e32 = default_engine()
    e64 = Engine(e32.device, precision="fp64")
    rep = tally_precision(W.plain_mc(), W.PLAIN_MC_GRID, 1_000_000, 42, engine32=e32, engine64=e64)
    for tally in ("kerma", "h10"):
        r = rep[tally]
        assert r["voxels"] > 10_000
        assert r["sigma_median"] < 0.05, (tally, r)
        assert r["total_rel"] < 1e-3, (tally, r)
    for k in ("fraction_absorbed", "fraction_escaped"):
        assert abs(rep[k]["fp32"] - rep[k]["fp64"]) < 2e-4, rep[k]
    # and the room scene, whose largest coordinate (300 cm) costs FP32 the most
    rep = tally_precision(W.room(), W.ROOM_GRID, 2_000_000, 7, engine32=e32, engine64=e64)
    for tally in ("kerma", "h10"):
        assert rep[tally]["sigma_median"] < 0.05, (tally, rep[tally])
        assert rep[tally]["total_rel"] < 2e-3, (tally, rep[tally])
