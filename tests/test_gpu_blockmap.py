"""Device BlockMap (blockmap.rs:35-209) against the crate's observable
semantics, restated as a Python dict: insert (later value wins), update as a
counter, get, remove with tombstones, sorted_pairs, growth by doubling at 3/4
load, and sentinel keys rejected."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_insert_get_sorted_pairs(msbg, ctx):
    r = np.random.default_rng(1)
    m = msbg.BlockMap(ctx)
    ref = {}
    for batch in range(6):
        keys = r.integers(0, 1 << 40, 5000).astype(np.uint64)
        keys[:500] = keys[500:1000]  # repeated keys in the batch: the later value wins
        vals = r.integers(0, 1 << 32, 5000).astype(np.uint32)
        m.insert(keys, vals)
        for k, v in zip(keys.tolist(), vals.tolist()):
            ref[k] = v
    assert len(m) == len(ref)
    k, v = m.sorted_pairs()
    want = sorted(ref.items())
    assert k.tolist() == [a for a, _ in want] and v.tolist() == [b for _, b in want]
    q = np.concatenate([k[:1000], r.integers(0, 1 << 40, 1000).astype(np.uint64)])
    got = m.get(q, missing=7)
    assert got.tolist() == [ref.get(x, 7) for x in q.tolist()]
    # with_capacity(4) then doubling: the smallest power of two holding len at 3/4
    cap = 4
    while len(ref) > cap * 3 // 4:
        cap *= 2
    assert m.capacity() >= cap


def test_update_add_is_a_histogram(msbg, ctx):
    r = np.random.default_rng(2)
    bids = r.integers(0, 3000, 200000).astype(np.uint64)
    m = msbg.BlockMap(ctx, 16)
    m.update_add(bids[:100000])
    m.update_add(bids[100000:])
    k, c = m.sorted_pairs()
    uk, uc = np.unique(bids, return_counts=True)
    assert np.array_equal(k, uk) and np.array_equal(c, uc.astype(np.uint32))


def test_remove_and_reinsert(msbg, ctx):
    r = np.random.default_rng(3)
    m = msbg.BlockMap(ctx)
    keys = np.arange(0, 40000, 3, dtype=np.uint64)
    m.insert(keys, (keys * 2).astype(np.uint32))
    gone = keys[::2]
    m.remove(gone)
    ref = {int(k): int(k) * 2 for k in keys}
    for g in gone.tolist():
        del ref[g]
    assert len(m) == len(ref)
    # re-insert some removed keys and overwrite some live ones: no key twice
    again = np.concatenate([gone[:1000], keys[1::2][:1000]])
    m.insert(again, np.full(len(again), 5, np.uint32))
    for g in again.tolist():
        ref[g] = 5
    k, v = m.sorted_pairs()
    assert len(k) == len(ref) == len(m) and len(np.unique(k)) == len(k)
    assert dict(zip(k.tolist(), v.tolist())) == ref
    assert m.get(gone[1000:1010], missing=9).tolist() == [9] * 10


def test_sentinel_keys_rejected(msbg, ctx):
    m = msbg.BlockMap(ctx)
    with pytest.raises(msbg.MsbgError):
        m.insert(np.array([2**64 - 1], np.uint64), np.array([1], np.uint32))
    with pytest.raises(msbg.MsbgError):
        m.update_add(np.array([1, 2**64 - 2], np.uint64))
    assert len(m) == 0


@pytest.mark.parametrize("blocks_per_axis", [16, 4096])  # dense table, and hash only (> 2^24 blocks)
def test_grid_ensure_blocks_device(msbg, ctx, blocks_per_axis):
    """ensure_blocks_parallel from a device list: new blocks hold the empty
    value, existing blocks keep their data, full dummies become value blocks,
    duplicates are allocated once, and the returned slots are the table's."""
    import torch
    s = 16 * blocks_per_axis
    g = msbg.SparseGrid(ctx, s, s, s, 0.25, 0.75, 16)
    r = np.random.default_rng(blocks_per_axis)
    nb = g.n_blocks
    first = np.unique(r.integers(0, nb, 300)).astype(np.uint64)
    g.write_blocks(first, r.uniform(-1, 1, (len(first), 4096)).astype(np.float32))
    before = g.read_blocks(first)
    full = np.setdiff1d(np.unique(r.integers(0, nb, 50)).astype(np.uint64), first)[:10]
    g.set_full_blocks(full)
    for rnd in range(3):
        batch = np.concatenate([first[:100], full, r.integers(0, nb, 2000).astype(np.uint64)])
        batch = np.concatenate([batch, batch[:500]])  # duplicates
        d = torch.from_numpy(batch.view(np.int64)).cuda()
        slots = torch.empty(len(batch), dtype=torch.int32, device="cuda")
        g.ensure_blocks_device(d, slots)
        ctx.synchronize()
        ids = np.sort(g.value_block_ids())
        want = np.union1d(np.union1d(first, full), batch)
        if rnd == 0:
            expected = want
        else:
            expected = np.union1d(expected, want)
        assert np.array_equal(ids, expected)
        assert np.array_equal(slots.cpu().numpy(), g.slots(batch))
    assert np.array_equal(g.read_blocks(first), before)
    fresh = np.setdiff1d(expected, first)
    assert np.all(g.read_blocks(fresh) == np.float32(0.25))
