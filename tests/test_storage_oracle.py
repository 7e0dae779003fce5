"""Storage element types in the oracle: binary16, Density8 and the lane
generator of the stochastic store (channel.rs:155-190, stencil.rs:103-192).

binary16 is pinned against numpy's IEEE round-to-nearest-even conversion;
the generator against the reference's own tests (stencil.rs:197-217: draws in
[0, 1), distinct seeds give distinct streams) and against the closed form the
device evaluates (state after k draws = lane seed * 16807^k mod 2^32); the
Density8 store against hand-worked cases of stencil.rs:176-192."""
import numpy as np
import pytest


def test_f16_conversion_matches_numpy(oracle):
    r = np.random.default_rng(0)
    mags = np.float32(10.0) ** r.integers(-9, 6, 100000).astype(np.float32)
    x = np.concatenate([r.standard_normal(100000).astype(np.float32) * mags,
                        np.array([0, -0.0, 1, 65504, 65519.99, 65520, 65536, 1e9, -1e9, 2.0 ** -24, 2.0 ** -25,
                                  3 * 2.0 ** -25, 2.0 ** -14, 6.1e-5, np.inf, -np.inf], np.float32)])
    with np.errstate(over="ignore"):
        want = x.astype(np.float16).view(np.uint16)
    assert np.array_equal(oracle.f32_to_f16(x), want)
    bits = np.arange(65536, dtype=np.uint32).astype(np.uint16)
    f = bits.view(np.float16).astype(np.float32)
    g = oracle.f16_to_f32(bits)
    assert np.all((f.view(np.uint32) == g.view(np.uint32)) | (np.isnan(f) & np.isnan(g)))


def lane_seed(seed, lane):
    """SimdRng::seed (stencil.rs:108-121) for one lane."""
    m = 0xFFFFFFFF
    h = (seed ^ (lane * 0x9E3779B9)) & m
    h ^= h >> 16
    h = (h * 0x85EBCA6B) & m
    h ^= h >> 13
    h = (h * 0xC2B2AE35) & m
    h ^= h >> 16
    return h if h else 0xDEADBEEF


@pytest.mark.parametrize("lanes", [4, 8, 16])
def test_lane_generator(oracle, lanes):
    u = oracle.lane_rng(0x12345678, lanes, 100)
    assert np.all((u >= 0) & (u < 1))  # stencil.rs:201-210
    assert not np.array_equal(oracle.lane_rng(1, lanes, 1), oracle.lane_rng(2, lanes, 1))  # :212-217
    # random access: draw k of lane l from seed_l * 16807^(k+1) mod 2^32
    for k in [0, 1, 17, 99]:
        for lane in range(lanes):
            st = (lane_seed(0x12345678, lane) * pow(16807, k + 1, 1 << 32)) & 0xFFFFFFFF
            f = np.array([(st >> 9) | 0x3F800000], np.uint32).view(np.float32)[0] - np.float32(1.0)
            assert u[k, lane] == f


def test_density8_store_known_answers(oracle):
    # sqrt(0.25) * 255 = 127.5: floor 127, fraction 0.5 -> 128 when u < 0.5
    v = np.array([0.25, 0.25, 1.0, 0.0, 0.0, 1.0001, -0.1, np.nan, 0.5], np.float32)
    u = np.array([0.4, 0.6, 0.99, 0.0, 0.999, 0.0, 0.5, 0.5, 0.0], np.float32)
    got = oracle.density8_store_sr(v, u)
    # 1.0001: sqrt * 255 = 255.01 -> 256 wraps to 0 in the u8 cast; -0.1 and
    # NaN: the x86 conversion's INT_MIN, whose low byte is 0
    sq = np.float32(np.sqrt(np.float32(0.5))) * np.float32(255.0)  # 180.31...
    assert list(got) == [128, 127, 255, 0, 0, 0, 0, 0, int(np.floor(sq)) + 1]


def test_density8_stream_continues_across_calls(msbg, oracle):
    """Two calls of one sweeper (2 + 1 sweeps) equal one call of 3."""
    r = np.random.default_rng(3)

    def grid():
        g = msbg.HostGrid("d8", 32, 32, 32, 0.0, 1.0, 16, "u8")
        for b in range(g.n_blocks):
            if b != 5:
                g.ensure_block(b)
                g.blocks[b][:] = r.integers(0, 256, g.N)
        return g

    a = grid()
    b = a.copy()
    active = list(a.blocks)
    pos = oracle.sweep_stochastic(a, active, 1, 0.05, 2, True, 99, 8, 0)
    assert pos == 2 * 7 * 4096 // 8
    pos = oracle.sweep_stochastic(a, active, 1, 0.05, 1, True, 99, 8, pos)
    assert oracle.sweep_stochastic(b, active, 1, 0.05, 3, True, 99, 8, 0) == pos
    for k in active:
        assert np.array_equal(a.blocks[k], b.blocks[k])
