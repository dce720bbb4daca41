"""Test helpers: ghost lists of a uniform periodic grid in the layout of
gbfk_ghost_csr (488 rows per block in BlockLab::load order,
MRAG/MRAGcore/MRAGBlockLab.h:256-279), with the blocks in arbitrary pool
slots."""
import numpy as np

BS = 8
LAB_GHOSTS = 488


def ghost_positions():
    """Lab positions (x, y, z) in [-1, 9)^3 of the 488 ghosts, in BlockLab order."""
    out = []
    for icode in range(27):
        if icode == 13:
            continue
        code = (icode % 3 - 1, (icode // 3) % 3 - 1, (icode // 9) % 3 - 1)
        s = [(-1 if c < 0 else 0) if c < 1 else BS for c in code]
        e = [(0 if c < 0 else BS) if c < 1 else BS + 1 for c in code]
        for z in range(s[2], e[2]):
            for y in range(s[1], e[1]):
                for x in range(s[0], e[0]):
                    out.append((x, y, z))
    assert len(out) == LAB_GHOSTS
    return np.array(out)


def uniform_topology(bpd: int, slots=None, padded_rows=()):
    """Blocks and ghost CSR of a uniform periodic bpd^3 grid.

    ``slots[b]`` is the pool slot of block b = bx + bpd*(by + bpd*bz).
    Rows listed in ``padded_rows`` (global row ids) get a second entry of
    weight 0 from another cell, which leaves the ghost value unchanged but
    makes the face go through the ghost-fill path instead of the direct
    neighbour read."""
    nb = bpd ** 3
    slots = np.arange(nb) if slots is None else np.asarray(slots)
    n = bpd * BS
    pos = ghost_positions()
    blocks = []
    src = np.empty(nb * LAB_GHOSTS, dtype=np.int64)
    for bz in range(bpd):
        for by in range(bpd):
            for bx in range(bpd):
                b = bx + bpd * (by + bpd * bz)
                blocks.append((int(slots[b]), 0, (bx, by, bz), 1.0 / n))
                g = np.stack([bx * BS + pos[:, 0], by * BS + pos[:, 1], bz * BS + pos[:, 2]], 1) % n
                sb = (g[:, 0] // BS) + bpd * ((g[:, 1] // BS) + bpd * (g[:, 2] // BS))
                cell = (g[:, 0] % BS) + BS * ((g[:, 1] % BS) + BS * (g[:, 2] % BS))
                src[b * LAB_GHOSTS:(b + 1) * LAB_GHOSTS] = slots[sb] * 512 + cell
    padded = set(int(r) for r in padded_rows)
    row_ptr = [0]
    s, w0 = [], []
    for r in range(nb * LAB_GHOSTS):
        s.append(src[r])
        w0.append(1.0)
        if r in padded:
            s.append(src[(r + 7) % src.size])
            w0.append(0.0)
        row_ptr.append(len(s))
    w0 = np.array(w0)
    csr = {"row_ptr": np.array(row_ptr, dtype=np.int64), "src": np.array(s, dtype=np.int64),
           "w0": w0, "w1": np.ones_like(w0), "w2": np.ones_like(w0)}
    return blocks, csr


def face_rows(block: int, face: int):
    """Global row ids of the 64 ghosts of a face (0: x-, 1: x+, 2: y-, ...)."""
    pos = ghost_positions()
    d, plus = face // 2, face % 2
    c = BS if plus else -1
    others = [i for i in range(3) if i != d]
    sel = (pos[:, d] == c) & np.all((pos[:, others] >= 0) & (pos[:, others] < BS), axis=1)
    return block * LAB_GHOSTS + np.flatnonzero(sel)


def dense_to_pool(vol: np.ndarray, slots):
    """Scatter a dense n^3 volume into pool order (slot-major, 512 cells per slot)."""
    n = vol.shape[0]
    bpd = n // BS
    blocks = vol.reshape(bpd, BS, bpd, BS, bpd, BS).transpose(0, 2, 4, 1, 3, 5).reshape(bpd ** 3, 512)
    # blocks[bz*bpd*bpd + by*bpd + bx] is block b
    out = np.zeros((int(np.max(slots)) + 1, 512), dtype=vol.dtype)
    out[np.asarray(slots)] = blocks
    return out.ravel()


def pool_to_dense(pool: np.ndarray, slots, n: int):
    bpd = n // BS
    blocks = pool.reshape(-1, 512)[np.asarray(slots)]
    return blocks.reshape(bpd, bpd, bpd, BS, BS, BS).transpose(0, 3, 1, 4, 2, 5).reshape(n, n, n)
