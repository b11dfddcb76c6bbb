"""The library's bounded waits end instead of hanging: a block that holds TMEM
and waits on an mbarrier nothing ever arrives on (the tensor-core joins' wait
helper, 2 s) records the expiry, frees its TMEM and returns, and the device
stays usable -- a kNN build right after it succeeds."""
import ctypes as C
import time

import numpy as np
import pytest

from tagore_b200 import synth

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_device_stays_usable(capi):
    flag = C.c_int(0)
    t = time.perf_counter()
    capi.check(capi.lib().tagore_wait_selftest(C.byref(flag)))
    el = time.perf_counter() - t
    assert flag.value == 1
    assert 1.5 < el < 30.0  # the 2 s limit, plus launch and copy
    base, _ = synth.mixture("sift", 3000, 128, 8, 81)
    st = capi.gnn_descent_host(base, 16, 3)
    g = st.download(0).reshape(3000, 16)
    st.free()
    assert (g < 3000).all()
