"""CPU checks of the KMC selection restatement (oracle/kmc.py) on hand-worked cases of the
reference's loops (kmc/KineticMonteCarlo.cpp:147-199, 1151-1160), and of its rates against
the reference's own event record (kmc/Event.cpp, compiled unchanged)."""
import math

import numpy as np
import pytest

import oracle
from oracle import kmc as K


def test_first_running_sum_strictly_above_threshold():
    r = [1.0, 2.0, 3.0]                       # running sums 1, 3, 6
    assert K.select(r, 0.5, 0.5)[0] == 2      # threshold 3: 3 > 3 is false
    assert K.select(r, 0.49, 0.5)[0] == 1
    assert K.select(r, 0.0, 0.5)[0] == 0
    assert K.select(r, 0.999999, 0.5)[0] == 2
    ch, tot, dt = K.select(r, 0.5, 0.5)
    assert tot == 6.0
    assert abs(dt - math.log(2.0) / 6.0) < 1e-15


def test_empty_and_zero_rates():
    assert K.select([], 0.3, 0.3) == (-1, 0.0, 0.0)
    assert K.select([0.0, 0.0], 0.3, 0.3) == (-1, 0.0, 0.0)
    # zero-rate events are never chosen
    assert K.select([0.0, 5.0, 0.0], 0.0, 0.3)[0] == 1


def test_arrhenius_rates():
    es = np.array([1.0, 1.1, 2.0])
    em = np.array([0.5, 0.5, 0.5])
    r = K.rates(es, em, [1, 1, 0], 1e13, 600.0)
    beta = 1.0 / (K.K_BOLTZMANN * 600.0)
    assert abs(r[0] - 1e13 * math.exp(-0.5 * beta)) <= 1e-15 * r[0]
    assert abs(r[0] / r[1] - math.exp(0.1 * beta)) <= 1e-12 * r[0] / r[1]
    assert r[2] == 0.0


def test_selection_frequencies_follow_rates():
    rng = np.random.default_rng(0)
    r = np.array([1.0, 4.0, 0.0, 5.0])
    counts = np.zeros(4)
    for u in rng.random(20000):
        counts[K.select(r, u, 0.5)[0]] += 1
    assert counts[2] == 0
    assert np.allclose(counts / counts.sum(), r / r.sum(), atol=0.015)


def test_uniforms_are_numpy_philox():
    bg = np.random.Philox(key=np.array([11, 0], dtype=np.uint64),
                          counter=np.array([3, 0, 0, 0], dtype=np.uint64))
    raw = bg.random_raw(9)
    expect = np.array([(int(x) >> 11) * 2.0 ** -53 for x in raw])
    assert np.array_equal(K.uniforms(11, 3, 9), expect)


# barriers exactly representable in float (the reference's event record stores E_a as float)
FLOAT_EXACT_BARRIERS = [0.125, 0.5, 0.8125, 1.0, 1.25, 1.5, 2.0, 3.0]


@pytest.mark.skipif(not oracle.reference_available("event"),
                    reason="the reference's kmc/Event.cpp is not built (oracle/Makefile)")
@pytest.mark.parametrize("temperature", [300.0, 600.0, 1200.0])
def test_rates_match_the_reference_event(temperature):
    """oracle/kmc.rates against the reference's own Event::Event (kmc/Event.cpp:66-105),
    compiled unchanged: the same harmonic-TST rate for every barrier the float record holds
    exactly, and for any other barrier the reference's rate is the FP64 rate at float(E_a)."""
    beta = 1.0 / (K.K_BOLTZMANN * temperature)

    def close(ours, ref, ea):
        # exp(-E_a beta) turns a relative rounding of its argument into a relative error of
        # |E_a beta| times it (the reference is built with -Ofast, which may round beta
        # differently): a few ulp of the argument
        return abs(ours - ref) <= 1e-15 * max(1.0, ea * beta) * ref

    for ea in FLOAT_EXACT_BARRIERS:
        ref, stored = oracle.reference_event_rate(ea, 1e13, temperature)
        assert stored == ea
        ours = K.rates(np.array([ea]), np.array([0.0]), [1], 1e13, temperature)[0]
        assert close(ours, ref, ea)
    rng = np.random.default_rng(5)
    for ea in rng.uniform(0.2, 2.5, 20):
        ref, stored = oracle.reference_event_rate(ea, 1e13, temperature)
        assert stored == float(np.float32(ea)) and stored != ea
        ours = K.rates(np.array([stored]), np.array([0.0]), [1], 1e13, temperature)[0]
        assert close(ours, ref, stored)
