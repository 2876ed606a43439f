"""Mesh checks used by the Surface Nets tests: the reference test suite's topology analysis (Step6Tests.cs
AnalyzeMeshTopology, :616-713) and IndexedMesh's signed volume (Geometry/IndexedMesh.cs:95-118), restated."""
import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components


def topology(idx):
    """(open edges, non-manifold edges, unique edges, connected triangle components)."""
    t = np.asarray(idx, dtype=np.int64).reshape(-1, 3)
    nt = len(t)
    if nt == 0:
        return 0, 0, 0, 0
    a = np.concatenate([t[:, 0], t[:, 1], t[:, 2]])
    b = np.concatenate([t[:, 1], t[:, 2], t[:, 0]])
    tri = np.tile(np.arange(nt), 3)
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = lo * (int(t.max()) + 1) + hi
    order = np.argsort(key, kind="stable")
    ks, ts = key[order], tri[order]
    uniq, start, counts = np.unique(ks, return_index=True, return_counts=True)
    open_edges = int((counts == 1).sum())
    nonman = int((counts > 2).sum())
    # edges used twice must be traversed once in each direction (consistent orientation)
    dkey = a * (int(t.max()) + 1) + b
    twice = uniq[counts == 2]
    lo2, hi2 = twice // (int(t.max()) + 1), twice % (int(t.max()) + 1)
    dset = set(dkey.tolist())
    nonman += int(sum(1 for u, v in zip(lo2.tolist(), hi2.tolist()) if not ((u * (int(t.max()) + 1) + v) in dset and
                                                                         (v * (int(t.max()) + 1) + u) in dset)))
    # triangle adjacency through shared edges
    rows, cols = [], []
    for s, c in zip(start, counts):
        ids = ts[s:s + c]
        for i in range(c):
            for j in range(i + 1, c):
                rows.append(ids[i]); cols.append(ids[j])
    g = sp.coo_matrix((np.ones(len(rows)), (rows, cols)), shape=(nt, nt))
    ncomp, _ = connected_components(g, directed=False)
    return open_edges, nonman, len(uniq), int(ncomp)


def signed_volume(pos, idx):
    p = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    t = np.asarray(idx, dtype=np.int64).reshape(-1, 3)
    a, b, c = p[t[:, 0]], p[t[:, 1]], p[t[:, 2]]
    return float(np.sum(a * np.cross(b, c)) / 6.0)


def sphere_field(nx, ny, nz, centres, radius, h=1.0):
    """The reference tests' smooth ramp: clamp(0.5 + (R - d) / 2h, 0, 1) at voxel centres, float32."""
    z, y, x = np.meshgrid(np.arange(nz, dtype=np.float32), np.arange(ny, dtype=np.float32),
                          np.arange(nx, dtype=np.float32), indexing="ij")
    d = None
    for c in centres:
        dc = np.sqrt((x + np.float32(0.5) - np.float32(c[0])) ** 2 + (y + np.float32(0.5) - np.float32(c[1])) ** 2 +
                     (z + np.float32(0.5) - np.float32(c[2])) ** 2)
        d = dc if d is None else np.minimum(d, dc)
    v = np.clip(np.float32(0.5) + (np.float32(radius) - d) / np.float32(2.0 * h), 0.0, 1.0)
    return np.ascontiguousarray(v.astype(np.float32).reshape(-1))


def saddle_field(nx, ny, nz, seed=0, p=0.45):
    """A random field whose 0.5-level set is full of face saddles and corner kisses (exercises the
    well-composedness passes): seeded uniform values, a fraction p above the threshold."""
    rng = np.random.default_rng(seed)
    v = rng.random(nx * ny * nz).astype(np.float32)
    return np.where(rng.random(nx * ny * nz) < p, 0.5 + 0.5 * v, 0.5 * v).astype(np.float32)
