"""The attainable-bandwidth diagnostic (jv_stream_probe) on the GPU: every
supported footprint of read and written arrays, each array larger than L2,
runs and reports a rate of DRAM traffic below the HBM3e's nominal
7.7-8 TB/s plus measurement slack, and above a floor that a pass which
skipped its arrays would not need to be held to."""
import pytest

from conftest import pkg

pytestmark = pytest.mark.gpu

jv = pkg()


@pytest.mark.parametrize("nr,nw", [(1, 1), (2, 1), (10, 3), (12, 7), (14, 6), (25, 11)])
def test_stream_probe_rates(nr, nw):
    gbs = jv.stream_probe(nr, nw, 1 << 25, reps=3)  # 128 MiB per array
    assert 500.0 < gbs < 9000.0, gbs
