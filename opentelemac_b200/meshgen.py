"""Synthetic P1 triangle meshes and wave-equation coefficients.

These generate the inputs the solver is measured on: an n x n node grid on
the unit square, each quad split along one diagonal, interior nodes
jittered, and a per-element depth field h_e.  The wave-equation operator is
A = M + dt*g*h_e*K_e (mass matrix plus depth-weighted stiffness), assembled
by the library's on-device assembly (bief_assemble_wave_dev).

Node numbering is row-major (node (i, j) -> j*n + i, i along x); elements
are numbered quad by quad, two triangles per quad, both counter-clockwise.
Connectivity is returned 0-based with shape (nelem, 3); the Fortran-order
1-based IKLE(NELMAX,3) the C ABI takes is `ikle_fortran(ikle0)`.
"""
import numpy as np

DT = 1.0
GRAV = 9.81


def square_mesh(n, seed=12345, jitter=0.2):
    """n x n nodes on [0,1]^2; interior nodes moved by U(-jitter, jitter)*dx
    in x and y (one seeded generator, x then y draws).  Returns
    (x, y, ikle0) with ikle0 int32 (nelem, 3)."""
    if n < 2:
        raise ValueError("n >= 2 required")
    dx = 1.0 / (n - 1)
    ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
    x = (ii * dx).astype(np.float64).ravel()
    y = (jj * dx).astype(np.float64).ravel()
    interior = ((ii > 0) & (ii < n - 1) & (jj > 0) & (jj < n - 1)).ravel()
    rng = np.random.default_rng(seed)
    k = int(interior.sum())
    if k and jitter:
        jx = rng.uniform(-jitter, jitter, size=k) * dx
        jy = rng.uniform(-jitter, jitter, size=k) * dx
        x[interior] += jx
        y[interior] += jy
    qi, qj = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="xy")
    a = (qj * n + qi).ravel()           # (i, j)
    b = a + 1                           # (i+1, j)
    c = a + n + 1                       # (i+1, j+1)
    d = a + n                           # (i, j+1)
    t1 = np.stack([a, b, c], axis=1)
    t2 = np.stack([a, c, d], axis=1)
    ikle0 = np.empty((2 * a.size, 3), dtype=np.int32)
    ikle0[0::2] = t1
    ikle0[1::2] = t2
    return x, y, ikle0


def centroids(x, y, ikle0):
    return x[ikle0].mean(axis=1), y[ikle0].mean(axis=1)


def depth_smooth(x, y, ikle0):
    """h_e = 5 + 4 sin(2 pi x_c) cos(2 pi y_c) at the element centroid."""
    xc, yc = centroids(x, y, ikle0)
    return 5.0 + 4.0 * np.sin(2.0 * np.pi * xc) * np.cos(2.0 * np.pi * yc)


def element_neighbours(ikle0):
    """Edge neighbours of each element, -1 where none: (nelem, 3)."""
    ne = ikle0.shape[0]
    edges = np.concatenate([ikle0[:, [0, 1]], ikle0[:, [1, 2]], ikle0[:, [2, 0]]])
    edges.sort(axis=1)
    owner = np.tile(np.arange(ne), 3)
    key = edges[:, 0].astype(np.int64) * (int(ikle0.max()) + 1) + edges[:, 1]
    order = np.argsort(key, kind="stable")
    ks = key[order]
    nb = -np.ones((ne, 3), dtype=np.int64)
    slot = np.repeat(np.arange(3), ne)
    same = ks[1:] == ks[:-1]
    i0, i1 = order[:-1][same], order[1:][same]
    nb[owner[i0], slot[i0]] = owner[i1]
    nb[owner[i1], slot[i1]] = owner[i0]
    return nb


def depth_loguniform(ikle0, seed=4242, lo=0.5, hi=500.0, passes=3):
    """h_e log-uniform in [lo, hi] (seeded), then `passes` rounds of
    arithmetic averaging of each element with its edge neighbours."""
    rng = np.random.default_rng(seed)
    h = np.exp(rng.uniform(np.log(lo), np.log(hi), size=ikle0.shape[0]))
    nb = element_neighbours(ikle0)
    valid = nb >= 0
    cnt = 1.0 + valid.sum(axis=1)
    for _ in range(passes):
        s = h.copy()
        for k in range(3):
            m = valid[:, k]
            s[m] += h[nb[m, k]]
        h = s / cnt
    return h


def wave_coef(h, dt=DT, g=GRAV):
    """Per-element diffusion coefficient dt*g*h_e of A = M + dt*g*h_e*K_e."""
    return (dt * g) * np.asarray(h, dtype=np.float64)


def random_solution(npoin, seed=777):
    return np.random.default_rng(seed).uniform(-1.0, 1.0, size=npoin)


def ikle_fortran(ikle0, nelmax=None):
    """0-based (nelem, 3) -> Fortran IKLE(NELMAX,3): column-major, 1-based,
    as a flat int32 array of length 3*NELMAX."""
    ne = ikle0.shape[0]
    nelmax = ne if nelmax is None else nelmax
    out = np.zeros((3, nelmax), dtype=np.int32)
    out[:, :ne] = ikle0.T + 1
    return out.ravel()


def shuffled(x, y, ikle0, seed=99):
    """The same mesh with nodes and elements renumbered at random (and each
    element's vertices rotated), to exercise unstructured numbering."""
    rng = np.random.default_rng(seed)
    n = x.size
    perm = rng.permutation(n)          # new index -> old node
    inv = np.empty(n, dtype=np.int64)
    inv[perm] = np.arange(n)
    eperm = rng.permutation(ikle0.shape[0])
    ik = inv[ikle0[eperm]]
    rot = rng.integers(0, 3, size=ik.shape[0])
    ik = np.stack([ik[np.arange(ik.shape[0]), (rot + s) % 3] for s in range(3)], axis=1)
    return x[perm], y[perm], ik.astype(np.int32), perm, eperm


def mesh_size_for_npoin(npoin):
    return max(2, int(round(np.sqrt(npoin))))


def batch_sizes(ninst=256, lo=2000, hi=200000, seed=4):
    """Grid sizes (nodes per side) of the batched workload: node counts drawn
    log-uniformly in [lo, hi] with a seed, each rounded to a square grid."""
    rng = np.random.default_rng(seed)
    npo = np.exp(rng.uniform(np.log(lo), np.log(hi), ninst))
    return [mesh_size_for_npoin(v) for v in npo]


def batch_instance(k, n):
    """Instance k of the batched workload on an n x n grid: its own mesh
    seed, the smooth depth field and a random right-hand side.  Returns
    x, y, ikle0, coef, b."""
    x, y, ik = square_mesh(n, seed=1000 + k)
    coef = wave_coef(depth_smooth(x, y, ik))
    b = np.random.default_rng(k).uniform(-1, 1, x.size)
    return x, y, ik, coef, b


def boundary_faces(ikle0):
    """Boundary faces in boundary order: (elements, faces), face f joining
    local points f and f+1 mod 3.  Faces of counter-clockwise elements that
    have no neighbour run the boundary counter-clockwise; each loop is walked
    from its lowest-numbered node, loops in order of that node."""
    nb = element_neighbours(ikle0)
    be, bf = np.nonzero(nb < 0)
    start = ikle0[be, bf]
    end = ikle0[be, (bf + 1) % 3]
    by_start = {int(a): q for q, a in enumerate(start)}
    seen = np.zeros(be.size, dtype=bool)
    order = []
    for q0 in np.argsort(start, kind="stable"):
        if seen[q0]:
            continue
        q = int(q0)
        while not seen[q]:
            seen[q] = True
            order.append(q)
            q = by_start.get(int(end[q]), q)
    order = np.array(order, dtype=np.int64)
    return be[order].astype(np.int32), bf[order].astype(np.int32)


def segments(ikle0, npoin):
    """Segment numbering of a P1 mesh with the conventions of BIEF's STOSEG
    (stoseg.f:94-225): the boundary segments first, in boundary order
    (boundary_faces), with GLOSEG = (first, second) point of the face; then
    every other edge, numbered at its first face in (element, face) order,
    with GLOSEG ordered by node number.  Returns g1, g2 (0-based GLOSEG
    columns), eltseg and oriseg (3, nelem): the segment of each element face
    and 1 where GLOSEG(.,1) is the face's first point, else 2."""
    ik = np.asarray(ikle0, dtype=np.int64)
    ne = ik.shape[0]
    a = np.concatenate([ik[:, 0], ik[:, 1], ik[:, 2]])      # face-major: f*ne + e
    b = np.concatenate([ik[:, 1], ik[:, 2], ik[:, 0]])
    key = np.minimum(a, b) * int(npoin) + np.maximum(a, b)
    be, bf = boundary_faces(ikle0)
    bq = bf.astype(np.int64) * ne + be              # face index of each boundary segment
    bkeys = key[bq]
    # the other edges, numbered in order of their first face in scan order
    # (element outer, face inner)
    q = np.arange(3 * ne)
    scan = (q % ne) * 3 + q // ne
    other = ~np.isin(key, bkeys)
    ok, so = key[other], scan[other]
    idx = np.lexsort((so, ok))
    ks = ok[idx]
    # (a mesh whose every edge is on the boundary has no other edges)
    head = np.r_[True, ks[1:] != ks[:-1]] if ks.size else np.zeros(0, dtype=bool)
    first_scan, first_key = so[idx][head], ks[head]
    keys_sorted = first_key[np.argsort(first_scan, kind="stable")]
    g1 = np.concatenate([a[bq], keys_sorted // int(npoin)])
    g2 = np.concatenate([b[bq], keys_sorted % int(npoin)])
    allkeys = np.concatenate([bkeys, keys_sorted])
    order = np.argsort(allkeys, kind="stable")
    seg = order[np.searchsorted(allkeys[order], key)]
    eltseg = seg.reshape(3, ne)
    oriseg = np.where(a == g1[seg], 1, 2).reshape(3, ne)
    return (g1.astype(np.int32), g2.astype(np.int32), eltseg.astype(np.int32),
            oriseg.astype(np.int32))


def delaunay_mesh(npts, seed=2027):
    """Unstructured P1 mesh: the Delaunay triangulation of `npts` points
    (the unit square's corners, points along its edges and uniform random
    points inside), elements counter-clockwise.  Node valences and boundary
    shapes vary as in real meshes."""
    from scipy.spatial import Delaunay
    rng = np.random.default_rng(seed)
    nb = max(4, int(np.sqrt(npts)))
    t = np.sort(rng.uniform(0, 1, (4, nb)), axis=1)
    edge = np.concatenate([np.stack([t[0], np.zeros(nb)], 1), np.stack([np.ones(nb), t[1]], 1),
                           np.stack([t[2], np.ones(nb)], 1), np.stack([np.zeros(nb), t[3]], 1)])
    corners = np.array([[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0]])
    inner = rng.uniform(0.02, 0.98, (max(npts - 4 - 4 * nb, 0), 2))
    pts = np.concatenate([corners, edge, inner])
    tri = Delaunay(pts).simplices.astype(np.int64)
    p = pts[tri]
    area2 = ((p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1])
             - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1]))
    cw = area2 < 0
    tri[cw] = tri[cw][:, [0, 2, 1]]
    keep = np.abs(area2) > 1e-12
    return pts[:, 0].copy(), pts[:, 1].copy(), tri[keep].astype(np.int32)
