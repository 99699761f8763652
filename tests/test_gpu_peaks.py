"""The L2 read probe behind the roofline's second denominator (pt_measure_l2_bandwidth)."""
import pytest

from photon_b200 import abi, native

pytestmark = pytest.mark.gpu


def test_l2_read_bandwidth_is_above_hbm_copy_rate():
    """An L2-resident read runs faster than the HBM copy rate of a B200 (~6.5 TB/s read + write) and
    well below an impossible figure; two runs agree within a factor of two."""
    a = native.l2_read_bandwidth(0)
    b = native.l2_read_bandwidth(0, 16 << 20, 32)
    assert 6000.0 < a < 200000.0
    assert 0.5 < a / b < 2.0


@pytest.mark.parametrize("nbytes,reps", [(1 << 10, 8), (1 << 30, 8), (32 << 20, 0)])
def test_l2_probe_rejects_bad_sizes(nbytes, reps):
    with pytest.raises(native.PhotonError) as e:
        native.l2_read_bandwidth(0, nbytes, reps)
    assert e.value.code == abi.PT_ERR_INVALID
