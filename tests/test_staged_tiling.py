"""Host-side check of the tiling and pipeline arithmetic of the TMA-staged coarse-level product
(k_mg_apply_nodes_tma in mycel_b200/csrc/fp32_kernels.cu), restated from the kernel with its constants read
from the source: every node of a level is covered once, every staged read stays inside its stage and names the
node the thread-per-node gather reads, every box starts on a 16-byte boundary (TMA's rule for the innermost
coordinate), and the six-stage schedule issues each of the 27 boxes once, after the CTA barrier that follows the
last read of its stage's previous box, with the mbarrier parity the wait expects.

No GPU: this is the arithmetic a launch is checked against before it runs.
"""
import os
import re

import numpy as np
import pytest

SRC = os.path.join(os.path.dirname(__file__), "..", "mycel_b200", "csrc", "fp32_kernels.cu")


def _constants():
    src = open(SRC).read()
    out = {}
    for name in ("kS1Nodes", "kS1Box", "kS1Stages", "kS1Group", "kMgDofMaxNodes", "kMgCoarseMax"):
        m = re.search(r"constexpr\s+(?:int|int64_t)\s+" + name + r"\s*=\s*(\d+)", src)
        assert m, name
        out[name] = int(m.group(1))
    return out


C = _constants()


def _levels(nx, ny, nz):
    """The multigrid levels (element counts) as mg_levels forms them: halve rounding up until the level has at
    most kMgCoarseMax DOFs (at least two levels)."""
    out = [(nx, ny, nz)]
    d = (nx, ny, nz)
    while len(out) < 16:
        if len(out) >= 2 and 3 * (d[0] + 1) * (d[1] + 1) * (d[2] + 1) <= C["kMgCoarseMax"]:
            break
        if d == (1, 1, 1):
            break
        d = tuple((v + 1) // 2 for v in d)
        out.append(d)
    return out


def _check_level(nx, ny, nz):
    nodes, box = C["kS1Nodes"], C["kS1Box"]
    nx1, ny1, nz1 = nx + 1, ny + 1, nz + 1
    nn = nx1 * ny1 * nz1
    ns = (nn + 3) & ~3
    sxy = nx1 * ny1
    nblk = (nn + nodes - 1) // nodes
    b = np.arange(nblk, dtype=np.int64)[:, None]
    tid = np.arange(256, dtype=np.int64)[None, :]
    n0 = b * nodes
    n = n0 + tid
    act = (tid < nodes) & (n < nn)
    ts = np.where(tid < nodes, tid, 0)
    nc = np.where(act, n, 0)
    i, j, k = nc % nx1, (nc // nx1) % ny1, nc // sxy
    for nb in range(27):
        off = (nb % 3 - 1) + nx1 * ((nb // 3) % 3 - 1) + sxy * (nb // 9 - 1)
        first = n0 + (0 if nb >= 13 else off)
        xs, rem = first & ~3, first & 3
        assert np.all(xs % 4 == 0)                        # 16-byte aligned box start (floats)
        row = (nb - 13) * 9 if nb >= 13 else (13 - nb) * 9
        assert 0 <= row and row + 9 <= 9 * 14
        col = ts + rem
        assert col.min() >= 0 and col.max() < box        # inside the staged row, for all 256 threads
        want = n + (0 if nb >= 13 else off)
        assert np.all((xs + col == want) | ~act)         # the node the gather reads
        ui, uj, uk = i + nb % 3 - 1, j + (nb // 3) % 3 - 1, k + nb // 9 - 1
        mi, mj, mk = np.clip(ui, 0, nx), np.clip(uj, 0, ny), np.clip(uk, 0, nz)
        inside = act & (mi == ui) & (mj == uj) & (mk == uk)
        m = mi + nx1 * (mj + ny1 * mk)
        assert np.all((m < nn) | ~inside)
        if nb < 13:                                      # transposed block: staged at the gather's neighbour
            assert np.all((want == m) | ~inside)
        # a staged entry past the tensor's end is TMA's zero fill, one in [nn, ns) the zero padding
        assert np.all(xs + col < ns + box)
    assert np.all((3 * n + 2 < 3 * nn) | ~act)
    cover = np.zeros(nn, np.int64)
    np.add.at(cover, n[act], 1)
    assert np.all(cover == 1)


GRIDS = [(192, 96, 96), (160, 80, 40), (161, 81, 41), (256, 256, 8), (203, 67, 35), (80, 80, 80)]


@pytest.mark.parametrize("grid", GRIDS)
def test_staged_levels_cover_every_node_in_bounds(grid):
    staged = [d for d in _levels(*grid)[1:] if (d[0] + 1) * (d[1] + 1) * (d[2] + 1) > C["kMgDofMaxNodes"]]
    assert staged
    for d in staged:
        _check_level(*d)


def test_bridge_stages_its_first_level():
    lv = _levels(192, 96, 96)
    assert lv[1] == (96, 48, 48)
    assert 97 * 49 * 49 > C["kMgDofMaxNodes"]
    assert (25 * 25 * 49) <= C["kMgDofMaxNodes"]  # level 2 keeps the thread-per-DOF product


def test_stage_schedule():
    """Prologue: boxes 0 .. S-1. After group g (boxes G g .. G g + G - 1), when a later group reuses its
    stages: one CTA barrier, then boxes G g + S .. G g + S + G - 1. Box nb waits on stage nb % S with parity
    (nb / S) & 1, which must equal the number of earlier boxes of that stage mod 2; a box is issued only after
    the barrier following the group of the stage's previous box (its last readers)."""
    S, G = C["kS1Stages"], C["kS1Group"]
    assert S % G == 0 and 27 % G == 0
    issued_after = {}  # box -> index of the barrier it was issued after (-1: prologue)
    for nb in range(min(S, 27)):
        issued_after[nb] = -1
    barriers = []
    for g in range(27 // G):
        if G * (g + 1) + S - G < 27:
            barriers.append(g)
            for q in range(G):
                nb = G * g + S + q
                if nb < 27:
                    assert nb not in issued_after
                    issued_after[nb] = g
    assert sorted(issued_after) == list(range(27))
    for nb in range(27):
        prev = nb - S
        if prev >= 0:
            assert issued_after[nb] == prev // G  # after the barrier that ends the previous box's group
        assert (nb // S) & 1 == (sum(1 for q in range(nb) if q % S == nb % S)) & 1
    # the box a group waits on was issued before that group starts (no wait on an unissued box)
    for g in range(27 // G):
        for q in range(G):
            nb = G * g + q
            assert issued_after[nb] < g
