"""Lattice geometry restated from LatticeQM.jl (input construction for the workloads).

Coordinates follow ``src/modules/Structure/Lattices/type.jl:65-72``: ``basis``
is a 3x3 matrix whose first ``d=2`` columns are the Bravais vectors and whose
third column is e_z; ``coords`` is 3xN, fractional in the first two rows and
Cartesian z in the third; ``extra`` holds named extra coordinates
(``sublattice``, ``layer``).  Julia's ``Iterators.product`` runs its FIRST
factor fastest; every enumeration below keeps that order so atom and k
orderings match the reference.
"""
import math
import numpy as np

# src/modules/Structure/Geometries/2d.jl:64-66
A_TRI = np.array([[math.cos(math.pi / 6), math.cos(math.pi / 6)],
                  [-math.sin(math.pi / 6), math.sin(math.pi / 6)],
                  [0.0, 0.0]])
A_HEX = math.sqrt(3.0) * A_TRI

# special points (fractional), src/modules/Structure/Geometries/2d.jl:6-19
KDICT_SQ = ({"Γ": (0.0, 0.0), "X": (0.5, 0.0), "Y": (0.0, 0.5), "M": (0.5, 0.5)},
            ["Y", "Γ", "M", "X", "Γ"])
KDICT_TRI = ({"Γ": (0.0, 0.0), "K": (1 / 3, 2 / 3), "M": (0.5, 0.5), "K'": (2 / 3, 1 / 3),
              "M2": (0.0, 0.5), "M3": (0.5, 0.0), "Γ1": (1.0, -1.0)},
             ["Γ", "K", "M", "K'", "Γ", "M"])


def product_first_fastest(*ranges):
    """Julia ``Iterators.product`` order: first factor varies fastest."""
    out = [()]
    for r in ranges:
        out = [o + (x,) for x in r for o in out]
    return out


class Lattice:
    def __init__(self, A2, coords, extra=None, labels=(), kdict=KDICT_TRI):
        basis = np.eye(3)
        basis[:, :2] = A2
        self.basis = basis
        self.coords = np.array(coords, dtype=float).reshape(3, -1)
        n = self.coords.shape[1]
        self.labels = list(labels)
        self.extra = (np.zeros((0, n)) if extra is None
                      else np.array(extra, dtype=float).reshape(len(self.labels), n))
        self.kdict = kdict

    def copy(self):
        lat = Lattice(self.basis[:, :2].copy(), self.coords.copy(), self.extra.copy(),
                      list(self.labels), self.kdict)
        return lat

    @property
    def A(self):
        return self.basis[:, :2]

    @property
    def B(self):
        # dual basis B = A (A^T A)^{-1}, type.jl:289-293
        A = self.A
        return A @ np.linalg.inv(A.T @ A)

    @property
    def norb(self):
        return self.coords.shape[1]

    def positions(self):
        return self.basis @ self.coords

    def allpositions(self):
        return np.vstack([self.positions(), self.extra])

    def extracoord(self, name):
        return self.extra[self.labels.index(name)]

    def newdimension(self, name, values):
        # type.jl:398-404
        self.labels.append(name)
        self.extra = np.vstack([self.extra, np.asarray(values, float).reshape(1, -1)])
        return self


def square(a=1.0):
    # 2d.jl:44-49
    return Lattice(np.array([[a, 0.0], [0.0, a], [0.0, 0.0]]), np.zeros((3, 1)), kdict=KDICT_SQ)


def triangular(a=1.0):
    # 2d.jl:75-79
    return Lattice(a * A_TRI, np.zeros((3, 1)))


def triangular_supercell(a=1.0):
    # 2d.jl:87-93: 3-site triangular cell, basis a*A_tri*[[1,-1],[1,2]]
    S = np.array([[1.0, -1.0], [1.0, 2.0]])
    return Lattice(a * A_TRI @ S, np.array([[0, 1 / 3, -1 / 3], [0, 1 / 3, 2 / 3], [0, 0, 0]]),
                   [[1.0, 2.0, 3.0]], ["sublattice"])


def honeycomb(a=1.0):
    # 2d.jl:103-109 (NN distance = a)
    return Lattice(a * A_HEX, np.array([[0, 1 / 3], [0, 1 / 3], [0, 0]]), [[0.0, 1.0]],
                   ["sublattice"])


def honeycomb_AB(a=1.0, z=3.0):
    # 2d.jl:147-153 (AB / Bernal bilayer)
    return Lattice(a * A_HEX, np.array([[0, 1 / 3, 2 / 3, 1 / 3], [0, 1 / 3, 2 / 3, 1 / 3],
                                        [-z / 2, -z / 2, z / 2, z / 2]]),
                   [[0.0, 1.0, 1.0, 0.0]], ["sublattice"])


def honeycomb_BA(a=1.0, z=3.0):
    # 2d.jl:160-166
    return Lattice(a * A_HEX, np.array([[0, -1 / 3, 1 / 3, -1 / 3], [0, -1 / 3, 1 / 3, -1 / 3],
                                        [-z / 2, -z / 2, z / 2, z / 2]]),
                   [[0.0, 1.0, 0.0, 1.0]], ["sublattice"])


def kagome(a=1.0):
    """Kagome lattice: triangular Bravais basis with sites at 0, a1/2, a2/2.

    The reference has no kagome geometry; this uses its generic
    ``Lattice(basis, coords)`` constructor (type.jl:78) as the model
    definition for the batched three-model workload.
    """
    return Lattice(a * A_TRI, np.array([[0, 0.5, 0], [0, 0, 0.5], [0, 0, 0]]))


def supercellpoints(M, offset=math.sqrt(np.finfo(float).eps)):
    # supercell.jl:239-265 (supercellpoints)
    M = np.asarray(M, dtype=np.int64)
    n = int(round(abs(np.linalg.det(M))))
    Phi = np.linalg.inv(M)
    corners = M @ np.array(product_first_fastest(range(2), range(2))).T
    lo = corners.min(axis=1)
    hi = corners.max(axis=1)
    pts = []
    for x in product_first_fastest(*(range(l, h + 1) for l, h in zip(lo, hi))):
        x0 = Phi @ np.array(x, float)
        if np.all((x0 < 1 - offset) & (x0 >= -offset)):
            pts.append(x)
    assert len(pts) == n
    return np.array(pts, dtype=np.int64).T


def superlattice(lat, S):
    # supercell.jl:30-52
    S = np.asarray(S, dtype=np.int64)
    if S.ndim == 1:
        S = np.diag(S)
    if np.array_equal(S, np.eye(2, dtype=np.int64)):
        return lat.copy()
    pts = supercellpoints(S)
    blocks = []
    for v in pts.T:
        c = lat.coords.copy()
        c[:2] += v[:, None]
        blocks.append(c)
    coords = np.hstack(blocks)
    coords[:2] = np.linalg.inv(S) @ coords[:2]
    extra = np.hstack([lat.extra for _ in range(pts.shape[1])])
    kd = ({k: tuple(S.T @ np.array(p)) for k, p in lat.kdict[0].items()}, lat.kdict[1])
    return Lattice(lat.A @ S, coords, extra, list(lat.labels), kd)


def repeat_cells(lat, ranges):
    # supercell.jl:92-106 (repeat!)
    blocks_c, blocks_e = [], []
    for I in product_first_fastest(*ranges):
        c = lat.coords.copy()
        c[:2] += np.array(I, float)[:, None]
        blocks_c.append(c)
        blocks_e.append(lat.extra)
    lat.coords = np.hstack(blocks_c)
    lat.extra = np.hstack(blocks_e)
    return lat


def rotation2d(t):
    # Structure/rotate.jl:8
    return np.array([[math.cos(t), -math.sin(t)], [math.sin(t), math.cos(t)]])


def rotatecoordinates(lat, theta):
    # type.jl:366-375 then fractionalize! (type.jl:327-332)
    R = lat.positions()
    R[:2] = rotation2d(theta) @ R[:2]
    R[:2] = lat.B.T @ R
    lat.coords = R
    return lat


def crop2unitcell(lat, offset=math.sqrt(np.finfo(float).eps)):
    # supercell.jl:157-162 with inunitrange (supercell.jl:232)
    u = lat.coords[:2]
    keep = np.all((u < 1 - offset) & (u >= -offset), axis=0)
    lat.coords = lat.coords[:, keep]
    lat.extra = lat.extra[:, keep]
    return lat


def twistangle(n, m=1):
    # Lattices/twist.jl:46-49
    return math.acos((3.0 * n * n + 3 * n * m + m * m / 2.0) / (3.0 * n * n + 3 * n * m + m * m))


def moire_supercell(n, m=1):
    # Lattices/twist.jl:67-70
    assert math.gcd(n, m) == 1
    return np.array([[n, -n - m], [n + m, 2 * n + m]], dtype=np.int64)


def twist(lat1, lat2, n, z=3.0, m=1):
    """Commensurate twisted bilayer, Lattices/twist.jl:88-113,131-177."""
    alpha = twistangle(n, m)
    S = moire_supercell(n, m)
    # static layer (twist.jl:131-139)
    w = lat1.copy()
    w.coords[2] += z / 2
    bot = superlattice(w, S)
    bot.newdimension("layer", np.zeros(bot.norb))
    # rotated layer (twist.jl:154-177)
    w = lat2.copy()
    w.coords[2] += z / 2
    w.coords *= -1.0
    w.coords[:2] = np.mod(w.coords[:2], 1.0)
    top = superlattice(w, S)
    top.newdimension("layer", np.ones(top.norb))
    repeat_cells(top, [range(-1, 2), range(-1, 2)])
    rotatecoordinates(top, alpha)
    crop2unitcell(top)
    assert top.norb == lat2.norb * int(round(abs(np.linalg.det(S))))
    assert bot.labels == top.labels
    bot.coords = np.hstack([bot.coords, top.coords])
    bot.extra = np.hstack([bot.extra, top.extra])
    return bot


def lattice_reduce(A):
    # Lattices/neighbors.jl:56-73 (Lagrange reduction)
    b1, b2 = A[:, 0].astype(float), A[:, 1].astype(float)
    U = np.eye(2, dtype=np.int64)
    for _ in range(1000):
        if np.linalg.norm(b1) > np.linalg.norm(b2):
            b1, b2 = b2, b1
            U = U[:, ::-1].copy()
        mm = int(round(float(b1 @ b2) / float(b1 @ b1)))
        if mm == 0:
            break
        b2 = b2 - mm * b1
        U[:, 1] -= mm * U[:, 0]
    return np.column_stack([b1, b2]), U


def foldcell(points, A):
    """Wigner-Seitz fold of fractional points, foldcell.jl:20-67."""
    _, U = lattice_reduce(A)
    combos = [U @ np.array(x) for x in product_first_fastest(range(-1, 2), range(-1, 2))
              if any(v != 0 for v in x)]
    G = np.array(combos, float).T
    M = A.T @ A
    norms = [g @ M @ g for g in G.T]
    shift = True
    while shift:
        shift = False
        for i, g in enumerate(G.T):
            for j in range(points.shape[1]):
                p = points[:, j]
                dd = ((p - g / 2) @ M @ g) / norms[i]
                if dd > 0:
                    points[:, j] = p - math.ceil(dd) * g
                    shift = True
    return points


def honeycomb_twisted(N, a=1.0, z=3.0, fold=True):
    # Geometries/2d.jl:222-226 and _finalize_twisted! (2d.jl:190-194)
    lat = honeycomb(a)
    slat = twist(lat, lat, N, z=z, m=1)
    if fold:
        slat.coords[0] -= 1 / 3
        slat.coords[1] -= 1 / 3
        pts = slat.coords[:2].copy()
        foldcell(pts, slat.A)
        slat.coords[:2] = pts
    return slat


def _fold_twisted(slat):
    # _finalize_twisted! (2d.jl:190-194): foldPC! with shift [1/3, 1/3, 0]
    slat.coords[0] -= 1 / 3
    slat.coords[1] -= 1 / 3
    pts = slat.coords[:2].copy()
    foldcell(pts, slat.A)
    slat.coords[:2] = pts
    return slat


def _bernal_layer(stack, a, z):
    # 2d.jl:198-204
    lat = honeycomb_AB(a, z) if stack == "AB" else honeycomb_BA(a, z)
    lat.coords[2] += z / 2
    return lat


def honeycomb_twisted_ABBA(N, a=1.0, z=3.0):
    # 2d.jl:235-241
    return _fold_twisted(twist(_bernal_layer("AB", a, z), _bernal_layer("AB", a, z), N, z=z))


def honeycomb_twisted_ABAB(N, a=1.0, z=3.0):
    # 2d.jl:248-254
    return _fold_twisted(twist(_bernal_layer("AB", a, z), _bernal_layer("BA", a, z), N, z=z))


def getneighborcells(A, k=1, halfspace=True, innerpoints=False, excludeorigin=True):
    # Lattices/neighbors.jl:88-127
    A_red, U = lattice_reduce(A)
    n = math.ceil(math.sqrt(3) * (k + 1))
    IJ = np.array(product_first_fastest(range(-n, n + 1), range(-n, n + 1)), dtype=np.int64).T
    D = np.round(np.linalg.norm(A_red @ IJ, axis=0), 9)
    d = np.unique(D)
    sel = (D <= d[k]) if innerpoints else (D == d[k])
    vecs = [tuple(int(x) for x in U @ v) for v in IJ[:, sel].T]
    if not halfspace:
        return [v for v in vecs if not (excludeorigin and all(x == 0 for x in v))]
    seen, keep = set(), []
    for v in vecs:
        if all(x == 0 for x in v):
            if not excludeorigin:
                keep.append(v)
        elif v not in seen and tuple(-x for x in v) not in seen:
            keep.append(v)
            seen.add(v)
    return keep


def regulargrid(nk=100, dim=2):
    """Uniform k grid k=(i/nk1, j/nk1), first index fastest (Structure/grid.jl:42-54)."""
    n1 = int(math.floor(nk ** (1 / dim) + 1e-9))
    it = np.arange(n1) / n1
    return np.array(product_first_fastest(*([it] * dim)), dtype=float).T.copy()


def kpath(lat, num_points=100, named_path=None):
    """Equal-arc-length k path through special points (Paths/discretizepath.jl:3-33,
    Lattices/path.jl:53-63); returns fractional points, shape (2, num_points)."""
    pts_d, default = lat.kdict
    names = default if named_path is None else named_path
    B = lat.B
    P = [B @ np.array(pts_d[nm], float) for nm in names]
    diffs = [P[i] - P[i - 1] for i in range(1, len(P))]
    lens = [float(np.linalg.norm(dv)) for dv in diffs]
    diffs = [dv / ln if ln > 0 else np.zeros_like(dv) for dv, ln in zip(diffs, lens)]
    cum = np.concatenate([[0.0], np.cumsum(lens)])
    out = []
    for s in np.linspace(0.0, cum[-1], num_points):
        dels = s - cum
        for i in range(1, len(P)):
            if dels[i - 1] >= 0 and dels[i] <= 0:
                out.append(P[i - 1] + dels[i - 1] * diffs[i - 1])
                break
    X = np.array(out).T
    return (B @ np.linalg.inv(B.T @ B)).T @ X
