"""A single-level block layer for the block-AMR tests.

JANC's AMR step (``src/janc_v2/simulation/time_step/TVD_RK3.py:15-36``)
takes its blocks' ghost layers from the external ``jaxamr`` package
(``amr.get_ghost_block_data``, ``amr.update_external_boundary``), which is
not part of the JANC repository and not installed here.  This module plays
that part in the tests with semantics of its own: the blocks of one level
tile an ``nbx x nby`` rectangle (block ``b`` at block row ``b // nby``,
column ``b % nby``); a block's 3-cell ghost layers are the neighbouring
blocks' cells, and outside the rectangle the mirror image of the cells
inside (zero-gradient; corners included); ``update_external_boundary``
returns the new interiors unchanged (no coarser level is coupled in).

The golden fixtures run the reference's own AMR step with these functions
installed as ``jaxamr.amr``; the tests give the same functions (on torch
tensors) to ``janc_b200``'s AMR step.  Works on NumPy arrays and torch
tensors alike (indexing and reshapes only).
"""


def info(nbx, nby):
    """Block info of an nbx x nby tiling (the fields this layer reads)."""
    return {"number": nbx * nby, "nbx": nbx, "nby": nby}


def _is_torch(a):
    return type(a).__module__.startswith("torch")


def _stack(parts, like):
    if _is_torch(like):
        import torch
        return torch.stack(parts)
    import numpy as np
    return np.stack(parts)


def _index(n, like):
    """Padded-axis gather index: the mirror of the first / last 3 cells."""
    idx = [2 - j for j in range(3)] + list(range(n)) + [n - 1 - j for j in range(3)]
    if _is_torch(like):
        import torch
        return torch.tensor(idx, device=like.device)
    import numpy as np
    return np.array(idx)


def grid_from_blocks(blk, nbx, nby):
    """[nb][nf][bx][by] -> [nf][nbx bx][nby by]"""
    nb, nf, bx, by = blk.shape
    assert nb == nbx * nby
    g = blk.reshape(nbx, nby, nf, bx, by)
    g = g.permute(2, 0, 3, 1, 4) if _is_torch(blk) else g.transpose(2, 0, 3, 1, 4)
    return g.reshape(nf, nbx * bx, nby * by)


def blocks_from_grid(g, nbx, nby):
    """[nf][nbx bx][nby by] -> [nb][nf][bx][by]"""
    nf, X, Y = g.shape
    bx, by = X // nbx, Y // nby
    b = g.reshape(nf, nbx, bx, nby, by)
    b = b.permute(1, 3, 0, 2, 4) if _is_torch(g) else b.transpose(1, 3, 0, 2, 4)
    return b.reshape(nbx * nby, nf, bx, by)


def get_ghost_block_data(ref_blk_data, ref_blk_info):
    """Every block with its 3-cell ghost layers: [nb][nf][bx + 6][by + 6]."""
    nbx, nby = ref_blk_info["nbx"], ref_blk_info["nby"]
    nb, nf, bx, by = ref_blk_data.shape
    g = grid_from_blocks(ref_blk_data, nbx, nby)
    ix, iy = _index(g.shape[1], g), _index(g.shape[2], g)
    p = g[:, ix][:, :, iy]
    parts = []
    for b in range(nb):
        i, j = b // nby, b % nby
        parts.append(p[:, i * bx:i * bx + bx + 6, j * by:j * by + by + 6])
    return _stack(parts, ref_blk_data)


def update_external_boundary(level, blk_data, blk_data1, ref_blk_info):
    """The new block interiors as given (single level: nothing to couple)."""
    return blk_data1
