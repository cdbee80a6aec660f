"""Host side of the seeded workloads: the counter-based generator the device
initialisation shares with the host (SplitMix64), and the shapes of the seeded
initial fields."""

import math

import numpy as np

from BoundaryLayerDynamics import workloads as W


def test_splitmix64_known_answers():
    """The published SplitMix64 sequence from state 1234567 (Steele, Lea and Flood,
    OOPSLA 2014; the generator that seeds the xoshiro family): the output function
    of the states 1234567 + k * 0x9E3779B97F4A7C15."""
    states = np.uint64(1234567) + np.arange(5, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    got = [int(v) for v in W.splitmix64(states)]
    assert got == [6457827717110365317, 3203168211198807973, 9817491932198370423,
                   4593380528125082431, 16408922859458223821]


def test_seeded_fields_shapes_and_statistics():
    les = W.les_spec(32, 16, (2 * math.pi, math.pi, 1.0))
    u, v, w = W.seeded_initial_fields(les, seed=11)
    assert u.shape == (16, 32, 32) and w.shape == (15, 32, 32)
    # perturbations of +-10 % of the log-law profile
    p = W.seeded_profiles(les)["vel1"][0]
    assert np.all(np.abs(u / p[:, None, None] - 1) <= 0.1 + 1e-15)
    assert np.all(np.abs(v / p[:, None, None]) <= 0.1 + 1e-15)
    dns = W.dns_spec(16, 8)
    u, v, w = W.seeded_initial_fields(dns, seed=3)
    assert abs(np.std(v) / (0.05 * W.DNS_UC) - 1) < 0.1
    # another seed, another field; the same seed, the same field
    assert not np.array_equal(W.seeded_initial_fields(dns, seed=4)[1], v)
    assert np.array_equal(W.seeded_initial_fields(dns, seed=3)[1], v)
