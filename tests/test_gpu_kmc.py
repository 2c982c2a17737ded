"""KMC step on the GPU (akmc_kmc_*, akmc_events_dedup) against the FP64 oracle."""
import numpy as np
import pytest

from oracle import kmc as K

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed,counter,n", [(0, 0, 1), (7, 5, 13), (2**63 + 5, 2**64 - 3, 40),
                                            (123456789, 10**6, 4096)])
def test_uniforms_bitwise(gpu, seed, counter, n):
    from akmc_b200 import kmc
    u = kmc.uniforms(seed, counter, n).cpu().numpy()
    assert np.array_equal(u, K.uniforms(seed, counter, n))


@pytest.mark.parametrize("n", [1, 7, 1000])
def test_select_matches_oracle(gpu, n):
    import torch
    from akmc_b200 import kmc
    rng = np.random.default_rng(n)
    for trial in range(20):
        em = rng.normal(-460.0, 5.0, n)
        es = em + rng.uniform(0.1, 2.0, n)
        usable = (rng.random(n) > 0.2).astype(np.int32)
        u = rng.random(2)
        if trial == 0:
            u[1] = 0.0
        step, rate, cum = kmc.select(torch.tensor(es, device=gpu), torch.tensor(em, device=gpu),
                                     torch.tensor(usable, device=gpu), 1e13, 600.0,
                                     torch.tensor(u, device=gpu))
        r_o = K.rates(es, em, usable, 1e13, 600.0)
        ch, tot, dt = K.select(r_o, u[0], u[1])
        rate = rate.cpu().numpy()
        assert np.allclose(rate, r_o, rtol=2e-15, atol=0.0)
        if tot > 0:
            assert abs(step["total_rate"] - tot) <= 1e-14 * tot
            assert abs(step["dt"] - dt) <= 1e-14 * dt
        assert step["chosen"] == ch
        assert step["n_usable"] == int(usable.sum())
        if ch >= 0:
            assert step["barrier"] == es[ch] - em[ch]


def test_select_no_usable_event(gpu):
    import torch
    from akmc_b200 import kmc
    z = torch.zeros(3, dtype=torch.float64, device=gpu)
    step, _, _ = kmc.select(z, z, torch.zeros(3, dtype=torch.int32, device=gpu), 1e13, 600.0,
                            torch.tensor([0.5, 0.5], dtype=torch.float64, device=gpu))
    assert step["chosen"] == -1 and step["total_rate"] == 0.0 and step["dt"] == 0.0


def test_dedup_matches_oracle(gpu):
    import torch
    from akmc_b200 import kmc
    rng = np.random.default_rng(3)
    nat, n = 50, 12
    box = np.tile([12.0, 12.0, 12.0], (n, 1))
    base = [rng.uniform(0, 12, (nat, 3)) for _ in range(4)]
    pos, energy, group = [], [], []
    for i in range(n):
        k = i % 4
        p = base[k] + rng.normal(0, 0.01 if i >= 4 else 0.0, (nat, 3))   # repeats of 4 saddles
        if i == 9:
            p[0] += 0.5                                 # one atom far: not a duplicate
        if i == 10:
            p = p + 12.0                                # a periodic image: a duplicate
        pos.append(p)
        energy.append(-100.0 + k + (2e-4 if i >= 4 else 0.0))
        group.append(0 if i != 11 else 1)               # another basin: not compared
    pos = np.concatenate(pos)
    begin = np.arange(n, dtype=np.int64) * nat
    natoms = np.full(n, nat, np.int32)
    usable = np.ones(n, np.int32)
    usable[7] = 0
    group = np.array(group, np.int32)
    energy = np.array(energy)
    t = lambda a: torch.tensor(a, device=gpu)
    dup = kmc.dedup(t(group), t(usable), t(energy), t(pos), t(begin), t(natoms), t(box),
                    e_tol=1e-3, d_tol=0.1).cpu().numpy()
    ref = K.dedup(group, usable, energy, pos, begin, natoms, box, 1e-3, 0.1)
    assert np.array_equal(dup, ref)
    assert dup[4] == 0 and dup[9] == -1 and dup[10] == 2 and dup[11] == -1 and dup[7] == -1


@pytest.mark.skipif(not __import__("oracle").reference_available("event"),
                    reason="the reference's kmc/Event.cpp is not built (oracle/Makefile)")
def test_rates_match_the_reference_event(gpu):
    """akmc_kmc_select's FP64 rates against the reference's own Event::Event
    (kmc/Event.cpp:66-105, compiled unchanged) on barriers its float record holds exactly."""
    import torch

    import oracle
    from akmc_b200 import kmc
    ea = np.array([0.125, 0.5, 0.8125, 1.0, 1.25, 1.5, 2.0, 3.0])
    em = np.full(len(ea), -460.0)          # float-exact minima: E_saddle - E_min == E_a exactly
    for temperature in (300.0, 600.0, 1200.0):
        beta = 1.0 / (K.K_BOLTZMANN * temperature)
        _, rate, _ = kmc.select(torch.tensor(em + ea, device=gpu), torch.tensor(em, device=gpu),
                                torch.ones(len(ea), dtype=torch.int32, device=gpu), 1e13, temperature,
                                torch.tensor([0.5, 0.5], device=gpu))
        rate = rate.cpu().numpy()
        for k, e in enumerate(ea):
            ref, stored = oracle.reference_event_rate(e, 1e13, temperature)
            assert stored == e
            assert abs(rate[k] - ref) <= 1e-15 * max(1.0, e * beta) * ref
