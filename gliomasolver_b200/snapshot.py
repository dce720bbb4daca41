"""Host snapshots of a block pool, so that a long run can resume.

The reference keeps no restart state for the forward solve: its dumps are
VTK files and the UQ matrix (Glioma/Glioma_ReactionDiffusion.cpp:191-267).
A snapshot here holds what a resumed gbfk_rd_step needs to continue bit for
bit: the precision and capacity of the pool, its topology (a uniform grid's
blocks per dimension, or the leaves and ghost lists given to
gbfk_set_topology), p_w, p_g and phi of every used slot, and the caller's own
metadata (step count, time, coefficients ...).  Only the public pool calls
are used: download on save; set_uniform / set_topology and upload on restore.

    save_snapshot("run.snap.npz", pool, meta={"step": k, "t": t})
    ...
    snap = load_snapshot("run.snap.npz")
    pool = restore_pool(snap)
    pool.rd_step(Dw, Dg, rho, dt, nsteps - snap.meta["step"])
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field

import numpy as np

FORMAT = 1
FIELD_NAMES = ("p_w", "p_g", "phi")
BLOCK_CELLS = 512


@dataclass
class Snapshot:
    precision: str
    max_blocks: int
    blocks_per_dim: int | None              # uniform grid, else None
    blocks: list | None                     # [(slot, level, (ix, iy, iz), h)] of a ghost-list topology
    csr: dict | None                        # row_ptr, src, w0, w1, w2
    fields: dict                            # name -> slot-major values, 512 per slot
    meta: dict = field(default_factory=dict)


def _used_slots(snapshot_blocks, blocks_per_dim):
    if blocks_per_dim is not None:
        return int(blocks_per_dim) ** 3
    return 1 + max(int(b[0]) for b in snapshot_blocks)


def save_snapshot(path, pool, topology=None, meta=None):
    """Write ``pool``'s state to ``path`` (an .npz, replaced atomically).
    ``topology``: None for a pool set up with set_uniform, else the
    ``(blocks, csr)`` last given to its set_topology (the pool does not keep
    the host copy).  ``meta``: a JSON-serialisable dict stored with it."""
    if topology is None:
        if pool.n is None:
            raise ValueError("save_snapshot: the pool has a ghost-list topology; pass topology=(blocks, csr)")
        bpd, blocks, csr = pool.n // 8, None, None
    else:
        bpd, (blocks, csr) = None, topology
        if not blocks:
            raise ValueError("save_snapshot: empty topology")
    ncells = _used_slots(blocks, bpd) * BLOCK_CELLS
    arrays = {name: pool.download(name, ncells) for name in FIELD_NAMES}
    header = {"format": FORMAT, "precision": pool.precision, "max_blocks": int(pool.max_blocks),
              "blocks_per_dim": bpd, "meta": dict(meta or {})}
    if blocks is not None:
        arrays["block_slot"] = np.array([b[0] for b in blocks], dtype=np.int64)
        arrays["block_level"] = np.array([b[1] for b in blocks], dtype=np.int64)
        arrays["block_index"] = np.array([tuple(b[2]) for b in blocks], dtype=np.int64).reshape(-1, 3)
        arrays["block_h"] = np.array([b[3] for b in blocks], dtype=np.float64)
        for k, dt in (("row_ptr", np.int64), ("src", np.int64), ("w0", np.float64), ("w1", np.float64),
                      ("w2", np.float64)):
            arrays["csr_" + k] = np.ascontiguousarray(csr[k], dtype=dt)
    arrays["header"] = np.frombuffer(json.dumps(header).encode(), dtype=np.uint8)
    path = os.fspath(path)
    tmp = f"{path}.tmp{os.getpid()}"
    try:
        with open(tmp, "wb") as f:
            np.savez(f, **arrays)
        os.replace(tmp, path)
    finally:
        if os.path.exists(tmp):
            os.remove(tmp)


def load_snapshot(path) -> Snapshot:
    with np.load(os.fspath(path)) as z:
        header = json.loads(bytes(z["header"]).decode())
        if header.get("format") != FORMAT:
            raise ValueError(f"{path}: snapshot format {header.get('format')}, expected {FORMAT}")
        bpd = header["blocks_per_dim"]
        blocks = csr = None
        if bpd is None:
            blocks = [(int(s), int(lv), tuple(int(v) for v in ix), float(h)) for s, lv, ix, h in
                      zip(z["block_slot"], z["block_level"], z["block_index"], z["block_h"])]
            csr = {k: z["csr_" + k].copy() for k in ("row_ptr", "src", "w0", "w1", "w2")}
        fields = {name: z[name].copy() for name in FIELD_NAMES}
    dtype = np.float64 if header["precision"] == "f64" else np.float32
    ncells = _used_slots(blocks, bpd) * BLOCK_CELLS
    for name, a in fields.items():
        if a.dtype != dtype or a.size != ncells:
            raise ValueError(f"{path}: field {name} has {a.size} {a.dtype} values, expected {ncells} {dtype}")
    return Snapshot(header["precision"], int(header["max_blocks"]), bpd, blocks, csr, fields, header["meta"])


def restore_pool(snap: Snapshot, pool=None, device: int = 0, stream=None):
    """A pool holding ``snap``'s state: a new BlockPool of the snapshot's
    capacity and precision, or ``pool`` if given (it must match both)."""
    if pool is None:
        from .solver import BlockPool

        pool = BlockPool(snap.max_blocks, snap.precision, device=device, stream=stream)
    elif pool.precision != snap.precision or pool.max_blocks < _used_slots(snap.blocks, snap.blocks_per_dim):
        raise ValueError("restore_pool: the pool's precision or capacity does not fit the snapshot")
    if snap.blocks_per_dim is not None:
        pool.set_uniform(snap.blocks_per_dim)
    else:
        pool.set_topology(snap.blocks, snap.csr)
    for name in FIELD_NAMES:
        pool.upload(name, snap.fields[name])
    return pool
