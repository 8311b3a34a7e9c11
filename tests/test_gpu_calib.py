"""The random-read ceiling the heavy-step bound uses: a sane rate, and bad arguments refused."""
import pytest

import wukong_b200 as wk

pytestmark = pytest.mark.gpu


def test_random_read_ceiling(ctx):
    rate = ctx.measure_random_reads(1 << 30, iters=3)
    assert 1e9 < rate < 1e12
    with pytest.raises(wk.WukongError) as e:
        ctx.measure_random_reads(4096, iters=1)
    assert e.value.code == wk.E_BADARG
