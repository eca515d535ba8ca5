"""BD-rate of the learned form against the plain full search, measured with
real bits from the reference's own host encoder (CABAC, fixed QP 22/27/32/37)
and the PSNR of the reconstruction (tests/rd_harness.py), on a seeded
synthetic 720p sequence with pan, moving rectangles and a noise patch.

Bar: learned-form BD-rate <= 1.0 % (YUV PSNR) with at least half of the
searched MBs served from the network's candidates, and the packaged
checkpoint loads through the library's SHA-256 check."""
import os

import pytest

import rd_harness as rh

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bc250-vaapi_b200", "b200enc",
                       "data", "proposal_h264.b2pn")


@pytest.mark.skipif(not rh.available(), reason="reference integration not built")
@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="no packaged proposal checkpoint")
def test_learned_bdrate_within_one_percent(gpu):
    W, H = 1280, 720
    frames = rh.make_frames(W, H, 16, seed=77)
    curves = rh.rd_curves(gpu, frames, W, H, [rh.PLAIN, rh.LEARNED], conf=0.9)
    bd = rh.bd_rate(curves[rh.PLAIN], curves[rh.LEARNED])
    learned = sum(r["learned"] for r in curves[rh.LEARNED])
    fallback = sum(r["fallback"] for r in curves[rh.LEARNED])
    print(f"BD-rate learned vs plain: {bd:+.3f}%  learned MBs {learned}  fallback MBs {fallback}")
    assert bd <= 1.0
    assert learned >= fallback
