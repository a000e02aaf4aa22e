"""The library runs on a B200 with kernels built for it: the tensor-core
contraction kernel reports binary version 100 (sm_100a), and the device is a
compute capability 10.0 part."""
import pytest

import gccu

pytestmark = pytest.mark.gpu


def test_kernels_built_for_sm100a(built):
    e = gccu.Engine(0)
    try:
        cc, sms, binary, ptx = e.device_info()
    finally:
        e.close()
    assert cc == 100, cc
    assert binary == 100, binary
    assert ptx == 100, ptx
    assert sms >= 1
