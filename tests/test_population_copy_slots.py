"""The slot rule of the collision's population copy (k_collide_list), on the
CPU: the column pass appends each 32-cell column chunk's active cells together
and in k order to one of 64 shards, chunks in any order; the collision takes a
cell's rank in its chunk from the list entries just before it in the same
shard that lie between the chunk's first cell and the cell.  The rank found
that way is the true rank, so no two cells of one step share a slot
(((i*ny + j) * ceil(nz/32) + k/32) * 2 + rank, ranks 0 and 1)."""
import numpy as np

SHARDS = 64
DEPTH = 2


def build_lists(active, nx, ny, nz, rng):
    """Shard lists as the column pass appends them: a warp per column, one
    append per chunk with active cells, warps in a random order."""
    shards = [[] for _ in range(SHARDS)]
    chunks = []
    for col in range(nx * ny):
        for k0 in range(0, nz, 32):
            ks = [k for k in range(k0, min(k0 + 32, nz)) if active[col, k]]
            if ks:
                chunks.append((col, [col * nz + k for k in ks]))
    for idx in rng.permutation(len(chunks)):
        col, cells = chunks[idx]
        shards[col % SHARDS].extend(cells)
    return shards


def slot_of(shard, pos, nz):
    """The collision's rule for the entry at position pos of its shard."""
    c = shard[pos]
    k = c % nz
    chunk_lo = c - (k & 31)
    rk = 0
    while rk < DEPTH and rk < pos:
        e = shard[pos - 1 - rk]
        if e < chunk_lo or e >= c:
            break
        rk += 1
    if rk >= DEPTH:
        return None, rk
    col = c // nz
    return (col * ((nz + 31) // 32) + (k >> 5)) * DEPTH + rk, rk


def test_ranks_are_true_chunk_ranks_and_slots_unique():
    rng = np.random.default_rng(7)
    for nx, ny, nz in ((6, 5, 96), (4, 7, 70), (3, 3, 33)):
        for density in (0.05, 0.3, 0.9):
            active = rng.random((nx * ny, nz)) < density
            shards = build_lists(active, nx, ny, nz, rng)
            used = set()
            for shard in shards:
                for pos, c in enumerate(shard):
                    col, k = divmod(c, nz)
                    k0 = k - (k & 31)
                    true_rank = int(active[col, k0:k].sum())
                    slot, rk = slot_of(shard, pos, nz)
                    assert rk == min(true_rank, DEPTH)
                    if slot is not None:
                        assert slot not in used
                        used.add(slot)
                        assert 0 <= slot < nx * ny * ((nz + 31) // 32) * DEPTH
