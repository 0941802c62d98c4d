"""The oracle's restatement of AC1D::Calculate_AC_UW_Mapped's route choice
(IAC/AC1D.cpp:248-379), on the CPU: known answers for the self-pair quirk of
the host loop and the composition of the two per-frame routes."""
import numpy as np

from helpers import random_frames, small_detector


def _acuw(o, ph, off, npix, sh, interp, route):
    ac = np.zeros(sh.size, np.float64)
    o.lib().iaco_ac1d_uw_frames(o.p(np.ascontiguousarray(ph)), o.p(np.ascontiguousarray(off, np.uint64)),
                                len(off) - 1, int(npix), sh.max_q, sh.dq_per_step, sh.size, interp, route,
                                o.p(ac))
    return ac


def test_host_loop_counts_the_self_pair_twice(oracle_lib):
    """One photon of 3 counts: the host loop (k >= j, factor 2) puts 18 at
    bin 0, the device kernel (ordered pairs) 9."""
    o = oracle_lib
    sh = o.ac1d_shape([0.5, 0.4, 0.1], 64)
    ph = np.array([[0.1, 0.2, 0.9, 3.0]], np.float32)
    off = np.array([0, 1], np.uint64)
    for interp in (0, 1):
        host = _acuw(o, ph, off, 1000, sh, interp, 0)
        dev = _acuw(o, ph, off, 1000, sh, interp, 1)
        assert host[0] == 18.0 and dev[0] == 9.0
        assert host[1:].sum() == 0 and dev[1:].sum() == 0
        # 1 hit of 1000 pixels is below 0.75 %: the reference takes the host loop
        np.testing.assert_array_equal(_acuw(o, ph, off, 1000, sh, interp, -1), host)
        # 1 hit of 100 pixels is above: the device kernel
        np.testing.assert_array_equal(_acuw(o, ph, off, 100, sh, interp, -1), dev)


def test_route_choice_composes_the_two_routes(oracle_lib, rng):
    o = oracle_lib
    pm, km, mq = small_detector(20, 30, 8e-4)
    npix = 600  # 0.0075 * 600 = 4.5 hits
    ph, off = random_frames(km, [1, 3, 4, 5, 9, 30, 0, 2], rng, max_count=4)
    sh = o.ac1d_shape(mq, 97)
    for interp in (0, 1):
        want = np.zeros(sh.size)
        for f in range(len(off) - 1):
            a, b = int(off[f]), int(off[f + 1])
            sub_off = np.array([0, b - a], np.uint64)
            route = 0 if np.float32(b - a) / np.float32(npix) < np.float32(0.0075) else 1
            want += _acuw(o, ph[a:b], sub_off, npix, sh, interp, route)
        np.testing.assert_allclose(_acuw(o, ph, off, npix, sh, interp, -1), want, rtol=1e-13, atol=0)
