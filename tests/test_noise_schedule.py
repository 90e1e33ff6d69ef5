"""The work split of the device noise generator (polyswift_plusplus_b200/csrc/noise.cu),
restated in numpy and checked on the CPU against the oracle's sequential
MT19937 + polar Gaussians (psstd/PsRandom.h:327-364).

What is checked here is the schedule the kernels follow, not the kernels:
- the twist with one barrier per generation (thread t builds elements t,
  t + 227 and t + 454, thread 169 also builds 623) reproduces the sequential
  generator;
- ranking accepted pair attempts by a prefix count, writing pair q to outputs
  2q (+1 when a cached value is pending) and 2q + 1, and moving the state to
  just after the last pair used (index 624 at a generation's end) reproduce the
  sequential Gaussian stream and its position, over several iterations and
  for odd draw counts that leave a cached value.
The kernels themselves are checked against the oracle on the GPU
(test_gpu_parity.py::test_device_noise_follows_the_host_stream).
"""
import math

import numpy as np
import pytest

import oracle as O

UPPER, LOWER, MATRIX = np.uint32(0x80000000), np.uint32(0x7FFFFFFF), np.uint32(0x9908B0DF)


def twist(a, b, c):
    y = (a & UPPER) | (b & LOWER)
    return c ^ (y >> np.uint32(1)) ^ np.where(y & np.uint32(1), MATRIX, np.uint32(0))


def temper(y):
    y = y ^ (y >> np.uint32(11))
    y = y ^ ((y << np.uint32(7)) & np.uint32(0x9D2C5680))
    y = y ^ ((y << np.uint32(15)) & np.uint32(0xEFC60000))
    return y ^ (y >> np.uint32(18))


def seeded_state(seed):
    bg = np.random.MT19937(0)
    bg._legacy_seeding(seed)
    return bg.state["state"]["key"].astype(np.uint32)


def device_twist(mt, G):
    """rng_twist_kernel: the state words of generations 0..G, concatenated."""
    out = [mt]
    o = mt
    for _ in range(G):
        t = np.arange(227)
        a = twist(o[t], o[t + 1], o[t + 397])
        b = twist(o[t + 227], o[t + 228], a)
        c = twist(o[454:623], o[455:624], b[:169])
        a0 = twist(o[0], o[1], o[397])
        d = twist(o[623], a0, b[169])  # b[169] is new element 396
        o = np.concatenate([a, b, c, [d]]).astype(np.uint32)
        out.append(o)
    return np.concatenate(out)


def device_iteration(st, K, sigma):
    """One iteration of K draws: rng_count/scan/out/final on the state dict."""
    P = (K + 1) // 2 + 1
    need = math.ceil(P / 0.7853981) + 10 * math.ceil(math.sqrt(P)) + 64
    G = (2 * need + 623) // 624
    J = G * 312
    words = device_twist(st["mt"], G)
    pos = st["idx"] + 2 * np.arange(J)
    a = temper(words[pos]).astype(np.float64) * (1.0 / 4294967296.0)
    b = temper(words[pos + 1]).astype(np.float64) * (1.0 / 4294967296.0)
    v1, v2 = 2.0 * a - 1.0, 2.0 * b - 1.0
    r = v1 * v1 + v2 * v2
    acc = ~((r >= 1.0) | (r == 0.0))
    rank = np.cumsum(acc) - acc  # exclusive prefix count
    off = 1 if st["have"] else 0
    out = np.empty(K)
    if off:
        out[0] = sigma * st["gauss"]
    last = None
    for j in np.nonzero(acc)[0]:
        o1 = off + 2 * int(rank[j])
        if o1 >= K:
            break
        fac = math.sqrt(-2.0 * math.log(r[j]) / r[j])
        out[o1] = sigma * (v2[j] * fac)
        if o1 + 1 < K:
            out[o1 + 1] = sigma * (v1[j] * fac)
        if o1 == K - 1:
            last = (j, True, v1[j] * fac)
        elif o1 + 1 == K - 1:
            last = (j, False, 0.0)
    if K - off <= 0:
        st["have"] = False
        return out
    assert last is not None, "pair margin exceeded"
    j, have, g = last
    p = st["idx"] + 2 * (int(j) + 1)
    gen, idx = divmod(p, 624)
    if idx == 0:
        gen, idx = gen - 1, 624
    assert gen <= G
    st.update(mt=words[gen * 624:(gen + 1) * 624], idx=idx, have=have, gauss=g)
    st["consumed"] += p - st["start_idx"]
    st["start_idx"] = idx
    return out


def test_twist_schedule_matches_the_sequential_generator(oracle_lib):
    seed = 38383
    words = device_twist(seeded_state(seed), 6)
    # the stream after init_genrand is generations 1, 2, ... tempered
    assert np.array_equal(temper(words[624:]), O.mt_u32(seed, 6 * 624).astype(np.uint32))


@pytest.mark.parametrize("seed,counts", [(38383, [2000, 2000, 2000]), (7, [1, 1, 1, 3, 5, 2, 1001]),
                                         (91, [4097, 311, 624, 1249])])
def test_split_noise_stream_matches_the_sequential_gaussians(oracle_lib, seed, counts):
    st = dict(mt=seeded_state(seed), idx=624, have=False, gauss=0.0, consumed=0, start_idx=624)
    got = np.concatenate([device_iteration(st, K, 0.25) for K in counts])
    ref = 0.25 * O.mt_gauss(seed, sum(counts))
    assert np.array_equal(got, ref)
    # the state sits exactly where the sequential generator stands: its next
    # word is the next word of the stream
    nxt = st["mt"][st["idx"]] if st["idx"] < 624 else device_twist(st["mt"], 1)[624]
    assert temper(np.uint32(nxt)) == O.mt_u32(seed, st["consumed"] + 1)[-1]
    # an odd total leaves the second value of the last pair cached
    assert st["have"] == (sum(counts) % 2 == 1)
