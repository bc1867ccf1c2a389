"""CPU oracle: a numpy restatement of the reference's periodic KIFMM evaluation pass.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (the C-ABI library, its
CUDA kernels or the Python mirror of the reference interface) imports or
calls this module; only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` use it, and only
as the checker.

It restates, function by function, the ``3dpp`` variant of
mumairsadiq/exafmm-rd (every citation is ``path:line`` inside that project):

* octree ............ ``3dpp/src/tree.cpp:102-188`` (+ ``get_child_cell_x`` 195-219)
* interaction lists . ``3dpp/src/traverser.cpp:19-326``
* precompute ........ ``3dpp/src/kernel.cpp:1638-1849``
* P2M/M2M/M2L/L2L/L2P/P2P ``3dpp/src/kernel.cpp`` (precompute paths) driven
  as in ``3dpp/src/fmm.cpp:13-294``
* dipole correction . ``3dpp/src/kernel.cpp:1580-1596``
* comparison metric . ``3dpp/src/body.cpp:131-175``
* inputs ............ ``3dpp/src/body.cpp:98-129`` (glibc ``drand48`` restated)
* Ewald sum ......... ``3dpp/src/ewald.cpp``

Third-party pieces the reference links and this restatement replaces:
FFTW3 (unpinned; the r2c/c2r of ``kernel.cpp:1290-1369,1725-1750``) by
``numpy.fft.rfftn/irfftn`` (same half-spectrum layout, normalised inverse),
and LAPACK ``dgesvd_`` (``3dpp/src/mathfunc.cpp:81-110``) by
``numpy.linalg.svd``.

Parity pin: ``tests/test_oracle_kats.py`` checks this oracle against the
FMM energies the reference printed in its own published runs
(``3dpp/exp/slurm-*.out``; extracted to ``tests/golden/log_kats.json``).
"""
import math

import numpy as np

INV4PI = 1.0 / (4.0 * math.pi)


# ----------------------------------------------------------------------------
# inputs
# ----------------------------------------------------------------------------
class Drand48:
    """glibc ``srand48``/``drand48``: the 48-bit LCG x' = (a x + c) mod 2^48,
    a = 0x5DEECE66D, c = 0xB, seeded with x = (seed << 16) | 0x330E; each draw
    returns x' / 2^48 (POSIX drand48 family, as used by
    ``3dpp/src/body.cpp:102-110``)."""

    A = 0x5DEECE66D
    C = 0xB
    M = (1 << 48) - 1

    def __init__(self, seed):
        self.x = ((seed & 0xFFFFFFFF) << 16) | 0x330E

    def next(self):
        self.x = (self.A * self.x + self.C) & self.M
        return self.x / float(1 << 48)

    def draws(self, n):
        """n consecutive draws, vectorised with the jump-ahead formula
        x_{k+j} = a^j x_k + c (a^j - 1)/(a - 1) mod 2^48."""
        out = np.empty(n, dtype=np.float64)
        block = 4096
        aj = [1]
        cj = [0]
        for _ in range(block):
            aj.append((aj[-1] * self.A) & self.M)
            cj.append((cj[-1] * self.A + self.C) & self.M)
        aj = aj[1:]
        cj = cj[1:]
        pos = 0
        while pos < n:
            m = min(block, n - pos)
            x0 = self.x
            vals = [((aj[j] * x0 + cj[j]) & self.M) for j in range(m)]
            out[pos:pos + m] = np.array(vals, dtype=np.float64) / float(1 << 48)
            self.x = vals[-1]
            pos += m
        return out


def generate_random_bodies(n, r, offset=(0.0, 0.0, 0.0), seed=5, zero_netcharge=1):
    """``generate_random_bodies`` (``3dpp/src/body.cpp:98-129``): per body
    three draws x_d = u*2r - r, then q = u - 0.5; optionally subtract the mean
    charge.  Returns positions (n,3) and charges (n,) in input (idx) order."""
    u = Drand48(seed).draws(4 * n).reshape(n, 4)
    x = u[:, :3] * r * 2 - r + np.asarray(offset, dtype=np.float64)
    q = u[:, 3] - 0.5
    if zero_netcharge:
        q_avg = 0.0
        for v in q:            # sequential sum, as the reference accumulates
            q_avg += v
        q_avg /= n
        q = q - q_avg
    return x, q


# ----------------------------------------------------------------------------
# surfaces and the convolution grid
# ----------------------------------------------------------------------------
def surface_point_num(p):
    """``get_surface_point_num`` (``3dpp/include/surface.h:10-13``)."""
    return 6 * (p - 1) * (p - 1) + 2


def surface_index(p):
    """Integer lattice coordinates (i, j, k) of the boundary points of a
    p^3 cube, i outermost and k innermost (``surface.cpp:3-47`` dir=0, and the
    identical enumeration ``get_surface_conv_map`` ``surface.h:28-48``)."""
    idx = []
    for i in range(p):
        for j in range(p):
            for k in range(p):
                if i in (0, p - 1) or j in (0, p - 1) or k in (0, p - 1):
                    idx.append((i, j, k))
    return np.array(idx, dtype=np.int64)


def surface_points(p, r, x=(0.0, 0.0, 0.0)):
    """``get_surface_points`` (``3dpp/src/surface.cpp:3-47``)."""
    ijk = surface_index(p).astype(np.float64)
    unit = -1.0 + ijk * (2.0 / (p - 1))
    return unit * r + np.asarray(x, dtype=np.float64)


class ConvGrid:
    """``conv_grid_setting`` (``3dpp/include/surface.h:58-86``)."""

    def __init__(self, P, r):
        self.N = 2 * P - 1
        self.N3 = self.N ** 3
        self.N_freq = self.N * self.N * (self.N // 2 + 1)
        self.delta = 2 * r / (P - 1) * 1.05
        self.gsize = r * 2 * 1.05


def conv_grid_points(N, gmin, delta, offset):
    """``get_conv_grid`` (``3dpp/src/surface.cpp:49-67``), shaped (N,N,N,3)
    indexed [k][j][i] (x fastest)."""
    a = -gmin + np.arange(N) * delta
    z, y, x = np.meshgrid(a, a, a, indexing="ij")
    g = np.stack([x, y, z], axis=-1)
    return g - np.asarray(offset, dtype=np.float64)


def inv_r(d):
    """1/|d| with 1/0 -> 0 (``kernel.cpp:1550-1552``, ``1607-1609``)."""
    r = np.sqrt(np.sum(d * d, axis=-1))
    with np.errstate(divide="ignore"):
        out = np.where(r == 0, 0.0, 1.0 / np.where(r == 0, 1.0, r))
    return out


def p2p_matrix(x_src, x_tar):
    """``get_p2p_matrix`` (``3dpp/src/kernel.cpp:1535-1556``): (tar, src)."""
    return inv_r(x_tar[:, None, :] - x_src[None, :, :])


def child_center(x_par, r_par, octant, periodic=False):
    """``Tree::get_child_cell_x`` (``3dpp/src/tree.cpp:195-219``)."""
    x_par = np.asarray(x_par, dtype=np.float64)
    if not periodic:
        s = np.array([1 if octant & 4 else -1, 1 if octant & 2 else -1, 1 if octant & 1 else -1],
                     dtype=np.float64)
        return x_par + s * (r_par / 2)
    k = octant // 9 - 1
    j = (octant % 9) // 3 - 1
    i = octant % 3 - 1
    return x_par + np.array([i, j, k], dtype=np.float64) * (r_par * 2 / 3.0)


# ----------------------------------------------------------------------------
# tree
# ----------------------------------------------------------------------------
class Cells:
    """Struct-of-arrays form of ``Cell3`` (``3dpp/include/tree.h:9-47``)."""

    def __init__(self):
        self.octant = []
        self.depth = []
        self.r = []
        self.x = []
        self.coff = []
        self.cnum = []
        self.boff = []
        self.bnum = []

    def add(self, octant, depth, r, x, coff, cnum, boff, bnum):
        self.octant.append(octant)
        self.depth.append(depth)
        self.r.append(r)
        self.x.append(np.asarray(x, dtype=np.float64))
        self.coff.append(coff)
        self.cnum.append(cnum)
        self.boff.append(boff)
        self.bnum.append(bnum)
        return len(self.octant) - 1

    def __len__(self):
        return len(self.octant)

    def is_leaf(self, c):
        return self.cnum[c] == 0


def build_nonuniform_octree(x, center, r, ncrit):
    """``Tree::build_nonuniform_octree`` (``3dpp/src/tree.cpp:102-188``).

    Breadth-first; a cell splits while it holds more than ``ncrit`` bodies;
    octant = 4*(x>cx) + 2*(y>cy) + (z>cz); only non-empty children are made and
    they are stored contiguously; bodies are stably regrouped by octant.
    Returns (cells, perm) with perm[i] = input index of the i-th sorted body."""
    n = x.shape[0]
    perm = np.arange(n, dtype=np.int64)
    cells = Cells()
    cells.add(13, 0, r, center, 0, 0, 0, n)
    queue = [0]
    head = 0
    while head < len(queue):
        c = queue[head]
        head += 1
        if cells.bnum[c] > ncrit:
            b0 = cells.boff[c]
            nb = cells.bnum[c]
            seg = perm[b0:b0 + nb]
            cx = cells.x[c]
            pts = x[seg]
            code = ((pts[:, 0] > cx[0]).astype(np.int64) << 2) + \
                   ((pts[:, 1] > cx[1]).astype(np.int64) << 1) + \
                   (pts[:, 2] > cx[2]).astype(np.int64)
            order = np.argsort(code, kind="stable")
            perm[b0:b0 + nb] = seg[order]
            counts = np.bincount(code, minlength=8)
            nchild = int(np.count_nonzero(counts))
            insert = len(cells)
            cells.coff[c] = insert
            cells.cnum[c] = nchild
            off = b0
            for o in range(8):
                if counts[o] > 0:
                    k = cells.add(o, cells.depth[c] + 1, cells.r[c] / 2,
                                  child_center(cx, cells.r[c], o), 0, 0, off, int(counts[o]))
                    queue.append(k)
                    off += int(counts[o])
    return cells, perm


# ----------------------------------------------------------------------------
# traversal
# ----------------------------------------------------------------------------
class Traversal:
    """``Traverser`` (``3dpp/src/traverser.cpp``): P2P and M2L lists with
    periodic offsets, the image super-cells and the M2L parent map."""

    def __init__(self, cells, cycle, images):
        self.cells = cells
        self.p2p = {}            # target leaf -> [(source leaf, offset)]
        self.m2l = {}            # target -> [(source, offset)] (dual-walk M2L pairs)
        self.m2l_parent = {}     # target parent -> [(source parent, offset, is_single_parent)]
        self.images = images
        self.cycle = cycle
        self._traverse()

    # adjacency with the reference's 1.001 tolerance (traverser.cpp:314-326)
    def adjacent(self, a, b, off):
        c = self.cells
        dx = np.abs(c.x[a] - c.x[b] - off)
        dist = (c.r[a] + c.r[b]) * 1.001
        return bool(dx[0] <= dist and dx[1] <= dist and dx[2] <= dist)

    def neighbour(self, a, b, off):
        return self.adjacent(a, b, off) and self.cells.depth[a] == self.cells.depth[b]

    def horizontal_origin(self, tc, sc, tcp, scp, off):
        """``horizontal_origin`` (``traverser.cpp:70-148``), with an explicit
        stack instead of recursion; children are visited in the same order."""
        c = self.cells
        stack = [(tc, sc, tcp, scp)]
        while stack:
            tc, sc, tcp, scp = stack.pop()
            divide = 0
            if not self.adjacent(tc, sc, off):
                if self.adjacent(tc, scp, off) and c.is_leaf(tc) and c.depth[scp] >= c.depth[tc]:
                    self.p2p.setdefault(tc, []).append((sc, off))
                elif self.adjacent(tcp, sc, off) and c.is_leaf(sc) and c.depth[tcp] >= c.depth[sc]:
                    self.p2p.setdefault(tc, []).append((sc, off))
                elif self.neighbour(tcp, scp, off):
                    self.m2l.setdefault(tc, []).append((sc, off))
                else:
                    if c.is_leaf(tc) and c.is_leaf(sc):
                        pass
                    elif not c.is_leaf(tc) and c.is_leaf(sc):
                        divide = 1
                    elif c.is_leaf(tc) and not c.is_leaf(sc):
                        divide = 2
                    else:
                        divide = 1 if c.r[tc] >= c.r[sc] else 2
            else:
                if c.is_leaf(tc) and c.is_leaf(sc):
                    self.p2p.setdefault(tc, []).append((sc, off))
                elif not c.is_leaf(tc) and c.is_leaf(sc):
                    divide = 1
                elif c.is_leaf(tc) and not c.is_leaf(sc):
                    divide = 2
                else:
                    divide = 1 if c.r[tc] >= c.r[sc] else 2
            if divide == 1:
                kids = [(c.coff[tc] + i, sc, tc, scp) for i in range(c.cnum[tc])]
                stack.extend(reversed(kids))
            elif divide == 2:
                kids = [(tc, c.coff[sc] + i, tcp, sc) for i in range(c.cnum[sc])]
                stack.extend(reversed(kids))

    def _nonleaf_neighbours(self, periodic_offsets):
        """``make_M2L_parent_map`` (``traverser.cpp:234-249``) and the periodic
        part of ``make_M2L_parent_map_i1`` (``251-282``), vectorised per target
        over all cells (same O(C^2) predicate, same list order)."""
        c = self.cells
        ncell = len(c)
        X = np.array(c.x)
        R = np.array(c.r)
        D = np.array(c.depth)
        nonleaf = np.array(c.cnum) > 0
        for j in range(ncell):
            if not nonleaf[j]:
                continue
            base = np.abs(X[j][None, :] - X)   # |x_j - x_i| (offset 0)
            dist = (R[j] + R) * 1.001
            ok = nonleaf & (D == D[j]) & np.all(base <= dist[:, None], axis=1)
            ok[j] = False
            for i in np.nonzero(ok)[0]:
                self.m2l_parent.setdefault(j, []).append((int(i), np.zeros(3), 0))
        if periodic_offsets is None:
            return
        for j in range(ncell):
            if c.depth[j] == -1 or not nonleaf[j]:
                continue
            for i in range(ncell):
                if not nonleaf[i] or D[i] != D[j]:
                    continue
                for off in periodic_offsets:
                    if self.neighbour(j, i, off):
                        self.m2l_parent.setdefault(j, []).append((i, off, 0))

    def _traverse(self):
        """``Traverser::traverse`` (``traverser.cpp:19-68``)."""
        c = self.cells
        cycle = self.cycle
        images = self.images
        if images == 0:
            self.horizontal_origin(0, 0, 0, 0, np.zeros(3))
            self._nonleaf_neighbours(None)
            return
        # horizontal_periodic_near (traverser.cpp:150-176): depth -1 super-cell
        cidx = c.add(13, -1, c.r[0] * 3, c.x[0], 0, 1, 0, c.bnum[0])
        for pz in (-1, 0, 1):
            for py in (-1, 0, 1):
                for px in (-1, 0, 1):
                    off = np.array([px, py, pz], dtype=np.float64) * cycle
                    self.horizontal_origin(0, 0, cidx, cidx, off)
        offsets = [np.array([px, py, pz], dtype=np.float64) * cycle
                   for pz in (-1, 0, 1) for py in (-1, 0, 1) for px in (-1, 0, 1)
                   if (px, py, pz) != (0, 0, 0)]
        self._nonleaf_neighbours(offsets)
        if images >= 2:
            # horizontal_periodic_far (traverser.cpp:178-232): depth -2..-images
            child = len(c) - 1
            for m in range(1, images):
                k = c.add(13, -1 - m, c.r[child] * 3, c.x[child], child, 1, 0, 0)
                child = k
            # image-level parent M2L entries (traverser.cpp:43-64)
            idx = len(c) - 1 - images
            for m in range(1, images):
                ci = idx + m
                for pz in (-1, 0, 1):
                    for py in (-1, 0, 1):
                        for px in (-1, 0, 1):
                            if (px, py, pz) != (0, 0, 0):
                                off = np.array([px, py, pz], dtype=np.float64) * c.r[ci] * 2
                                self.m2l_parent.setdefault(ci, []).append((ci, off, 1))


# ----------------------------------------------------------------------------
# precompute
# ----------------------------------------------------------------------------
def svd_pinv_factors(A):
    """``svd`` + ``pseudo_inverse`` (``3dpp/src/mathfunc.cpp:81-110,154-169``):
    A = U S V^T; singular values at or below 4e-16 * s_max are dropped."""
    U, s, VT = np.linalg.svd(A)
    smax = np.max(np.abs(s))
    sinv = np.where(s > smax * 4e-16, 1.0 / np.where(s > 0, s, 1.0), 0.0)
    return U, sinv, VT


def hash_rel(v):
    """``LaplaceKernel::hash`` (``3dpp/include/kernel.h:136-141``)."""
    signs = ((1 if v[0] < 0 else 0) << 2) + ((1 if v[1] < 0 else 0) << 1) + (1 if v[2] < 0 else 0)
    return abs(v[0]) * 1000 + abs(v[1]) * 100 + abs(v[2]) * 10 + signs


def relx(rng, minv):
    """``get_relx`` / ``get_relx_idx_map`` (``kernel.h:149-194``): offsets in
    [-rng, rng]^3 with some |component| >= minv, z outermost, x innermost."""
    out = []
    for k in range(-rng, rng + 1):
        for j in range(-rng, rng + 1):
            for i in range(-rng, rng + 1):
                if abs(i) >= minv or abs(j) >= minv or abs(k) >= minv:
                    out.append((i, j, k))
    return out


class Operators:
    """Operator tables built once at the root radius r0
    (``LaplaceKernel::precompute`` ``kernel.cpp:1638-1704`` and
    ``precompute_m2l`` ``1706-1849``)."""

    def __init__(self, P, r0, images):
        self.P = P
        self.r0 = r0
        self.images = images
        ns = surface_point_num(P)
        self.ns = ns
        x_check = surface_points(P, r0 * 2.95)
        x_equiv = surface_points(P, r0 * 1.05)
        e2c = p2p_matrix(x_equiv, x_check)
        U, sinv, VT = svd_pinv_factors(e2c)
        self.UT_p2m = U.T
        V = VT.T
        self.VSinv_p2m = V * sinv[None, :]
        self.m2m = []
        for o in range(8):
            xe = surface_points(P, r0 / 2 * 1.05, child_center(np.zeros(3), r0, o))
            G = p2p_matrix(xe, x_check)
            self.m2m.append(self.VSinv_p2m @ (self.UT_p2m @ G))
        self.m2m_img = []
        if images > 0:
            for o in range(27):
                xe = surface_points(P, r0 / 3 * 1.05, child_center(np.zeros(3), r0, o, True))
                G = p2p_matrix(xe, x_check)
                self.m2m_img.append(self.VSinv_p2m @ (self.UT_p2m @ G))
        self.l2l = [m.T.copy() for m in self.m2m]
        self.l2l_img = self.m2m_img[13].T.copy() if images > 0 else None
        self.UT_l2p = V.T            # transpose(V_p2m)
        self.VSinv_l2p = U * sinv[None, :]   # transpose(UT_p2m) * Sinv
        # M2L kernel spectra (precompute_m2l, kernel.cpp:1721-1769)
        grid = ConvGrid(P, r0)
        self.grid = grid
        rng = 4 if images >= 2 else 3
        offs = relx(rng, 2)
        self.gk_index = {hash_rel(v): n for n, v in enumerate(offs)}
        N = grid.N
        self.gk = np.empty((len(offs), N, N, N // 2 + 1), dtype=np.complex128)
        for n, v in enumerate(offs):
            rel = np.array(v, dtype=np.float64) * r0 * 2
            g = inv_r(conv_grid_points(N, grid.gsize, grid.delta, rel))
            self.gk[n] = np.fft.rfftn(g)
        # 8x8 sibling blocks per parent direction (kernel.cpp:1783-1811)
        dirs = relx(1, 1)
        self.dirs = dirs
        self.cc8 = np.zeros((26, 8, 8, N, N, N // 2 + 1), dtype=np.complex128)  # [d][isrc][itar]
        for d, v in enumerate(dirs):
            par_x = np.array(v, dtype=np.float64) * 2
            for isrc in range(8):
                xs = child_center(par_x, 1.0, isrc)
                for itar in range(8):
                    xt = child_center(np.zeros(3), 1.0, itar)
                    dx = tuple(int(t) for t in np.round(xs - xt))
                    h = hash_rel(dx)
                    if h in self.gk_index:
                        self.cc8[d, isrc, itar] = self.gk[self.gk_index[h]]
        # 1x27 image blocks (kernel.cpp:1813-1849)
        self.cc27 = None
        if images >= 2:
            self.cc27 = np.zeros((26, 27, N, N, N // 2 + 1), dtype=np.complex128)
            for d, v in enumerate(dirs):
                par_x = np.array(v, dtype=np.float64) * 3
                cnt = 0
                for pz in (-1, 0, 1):
                    for py in (-1, 0, 1):
                        for px in (-1, 0, 1):
                            sx = tuple(int(t) for t in np.round(par_x + np.array([px, py, pz])))
                            self.cc27[d, cnt] = self.gk[self.gk_index[hash_rel(sx)]]
                            cnt += 1
        # surface <-> grid index maps (kernel.cpp:1246-1259)
        ijk = surface_index(P)
        self.up_idx = (ijk[:, 2], ijk[:, 1], ijk[:, 0])
        d = ijk + (P - 1)
        self.down_idx = (d[:, 2], d[:, 1], d[:, 0])


# ----------------------------------------------------------------------------
# the evaluation pass
# ----------------------------------------------------------------------------
class FMM:
    """``LaplaceFMM`` (``3dpp/src/fmm.cpp``) with ``use_precompute`` = 1."""

    def __init__(self, x, q, P, ncrit, images, cycle, center=(0.0, 0.0, 0.0),
                 dipole_correction=0, divide_4pi=0, ops=None):
        self.x_in = np.asarray(x, dtype=np.float64)
        self.q_in = np.asarray(q, dtype=np.float64)
        self.P = P
        self.ncrit = ncrit
        self.images = images
        self.cycle = cycle
        self.r = cycle / 2
        self.center = np.asarray(center, dtype=np.float64)
        self.dipole_correction = dipole_correction
        self.divide_4pi = divide_4pi
        self.cells, self.perm = build_nonuniform_octree(self.x_in, self.center, self.r, ncrit)
        self.x = self.x_in[self.perm]
        self.q = self.q_in[self.perm]
        self.trav = Traversal(self.cells, cycle, images)
        self.ops = ops if ops is not None else Operators(P, self.r, images)
        ncell = len(self.cells)
        self.q_equiv = np.zeros((ncell, self.ops.ns))
        self.p_check = np.zeros((ncell, self.ops.ns))
        self.phi = np.zeros(len(self.q))
        self.grad = np.zeros((len(self.q), 3))

    # -- stages ---------------------------------------------------------------
    def leaves(self):
        return [c for c in range(len(self.cells)) if self.cells.is_leaf(c)]

    def nonleaf_at(self, depth):
        c = self.cells
        return [i for i in range(len(c)) if c.depth[i] == depth and c.cnum[i] > 0]

    def depth_range(self):
        return min(self.cells.depth), max(self.cells.depth)

    def p2m(self, charges=None, leaves=None):
        """``p2m_precompute`` (``kernel.cpp:332-371``); `leaves` restricts it
        (a sharded pass)."""
        c = self.cells
        q = self.q if charges is None else charges
        o = self.ops
        for leaf in (self.leaves() if leaves is None else leaves):
            b0, nb = c.boff[leaf], c.bnum[leaf]
            xc = surface_points(self.P, c.r[leaf] * 2.95, c.x[leaf])
            pc = p2p_matrix(self.x[b0:b0 + nb], xc) @ q[b0:b0 + nb]
            self.q_equiv[leaf] = (0.5 ** c.depth[leaf]) * (o.VSinv_p2m @ (o.UT_p2m @ pc))

    def m2m(self):
        """``LaplaceFMM::M2M`` (``fmm.cpp:111-150``) with ``m2m_precompute``
        (``kernel.cpp:395-404``) and ``m2m_img_precompute`` (``434-442``)."""
        c = self.cells
        o = self.ops
        dmin, dmax = self.depth_range()
        for depth in range(dmax, dmin, -1):
            for par in self.nonleaf_at(depth):
                if depth >= 0:
                    for k in range(c.cnum[par]):
                        ch = c.coff[par] + k
                        self.q_equiv[par] += o.m2m[c.octant[ch]] @ self.q_equiv[ch]
                else:
                    ch = c.coff[par]
                    for k in range(27):
                        self.q_equiv[par] += o.m2m_img[k] @ self.q_equiv[ch]

    def m2l(self, targets=None):
        """``m2l_fft_precompute_t`` (``kernel.cpp:1140-1397``) with the 8x8 and
        1x27 Hadamard stages (``1012-1138``); `targets` restricts the target
        parents (a sharded pass)."""
        c = self.cells
        o = self.ops
        N = o.grid.N
        dir_index = {hash_rel(v): n for n, v in enumerate(o.dirs)}
        srcs = sorted({s for lst in self.trav.m2l_parent.values() for (s, _, _) in lst})
        qk = {}
        for s in srcs:
            grid = np.zeros((8, N, N, N))
            for k in range(c.cnum[s]):
                ch = c.coff[s] + k
                slot = 0 if c.octant[ch] == 13 else c.octant[ch]
                grid[slot][o.up_idx] = self.q_equiv[ch]
            qk[s] = np.fft.rfftn(grid, axes=(1, 2, 3))
        for t in sorted(self.trav.m2l_parent):
            if targets is not None and t not in targets:
                continue
            lst = self.trav.m2l_parent[t]
            bydir = {}
            for (s, off, single) in lst:
                rv = (c.x[s] + off - c.x[t]) / (c.r[t] * 2)
                d = dir_index[hash_rel(tuple(int(v) for v in np.round(rv)))]
                bydir[d] = (s, single)
            pk = np.zeros((8, N, N, N // 2 + 1), dtype=np.complex128)
            for d, (s, single) in bydir.items():
                if single == 0:
                    pk += np.einsum("ijxyz,ixyz->jxyz", o.cc8[d], qk[s])
                else:
                    pk[0] += np.sum(o.cc27[d], axis=0) * qk[s][0]
            scale = (2.0 if c.depth[t] >= -1 else 3.0) ** (c.depth[t] + 1)
            for k in range(c.cnum[t]):
                ch = c.coff[t] + k
                slot = 0 if c.octant[ch] == 13 else c.octant[ch]
                g = np.fft.irfftn(pk[slot], s=(N, N, N), axes=(0, 1, 2))
                self.p_check[ch] += g[o.down_idx] * scale

    def l2l(self, parents=None):
        """``LaplaceFMM::L2L`` (``fmm.cpp:195-229``) with ``l2l_precompute``
        (``kernel.cpp:1419-1428``) / ``l2l_img_precompute`` (``1430-1435``);
        `parents` restricts it (a sharded pass)."""
        c = self.cells
        o = self.ops
        dmin, dmax = self.depth_range()
        for depth in range(dmin, dmax):
            for par in self.nonleaf_at(depth):
                if parents is not None and par not in parents:
                    continue
                if depth >= 0:
                    for k in range(c.cnum[par]):
                        ch = c.coff[par] + k
                        self.p_check[ch] += o.l2l[c.octant[ch]] @ self.p_check[par]
                else:
                    ch = c.coff[par]
                    self.p_check[ch] += o.l2l_img @ self.p_check[par]

    def l2p(self, leaves=None):
        """``l2p_precompute`` (``kernel.cpp:1458-1511``); `leaves` restricts it."""
        c = self.cells
        o = self.ops
        for leaf in (self.leaves() if leaves is None else leaves):
            b0, nb = c.boff[leaf], c.bnum[leaf]
            qd = (0.5 ** c.depth[leaf]) * (o.VSinv_l2p @ (o.UT_l2p @ self.p_check[leaf]))
            xe = surface_points(self.P, c.r[leaf] * 2.95, c.x[leaf])
            d = self.x[b0:b0 + nb][:, None, :] - xe[None, :, :]
            ir = inv_r(d)
            self.phi[b0:b0 + nb] += ir @ qd
            self.grad[b0:b0 + nb] -= np.einsum("ts,tsk->tk", (ir ** 3) * qd[None, :], d)

    def p2p(self, charges=None, targets=None):
        """``p2p_1toN_256`` (``kernel.cpp:258-311``) over ``P2P_map``
        (``fmm.cpp:259-294``); `targets` restricts the target cells."""
        c = self.cells
        q = self.q if charges is None else charges
        for t, lst in self.trav.p2p.items():
            if targets is not None and t not in targets:
                continue
            b0, nb = c.boff[t], c.bnum[t]
            xt = self.x[b0:b0 + nb]
            for (s, off) in lst:
                s0, ns = c.boff[s], c.bnum[s]
                d = xt[:, None, :] - (self.x[s0:s0 + ns] + off)[None, :, :]
                ir = inv_r(d)
                self.phi[b0:b0 + nb] += ir @ q[s0:s0 + ns]
                self.grad[b0:b0 + nb] -= np.einsum("ts,tsk->tk", (ir ** 3) * q[s0:s0 + ns][None, :], d)

    def dipole_correction_(self):
        """``dipole_correction`` (``kernel.cpp:1580-1596``), bodies in tree order.
        The dipole is taken about the box centre (the reference's box is
        centred at the origin, ``argument.cpp:61-62``).  Mode 1 is the
        reference's per-body form coef |mu|^2 / (N q_i); mode 2 (not in the
        reference) subtracts the surface term's potential coef mu . (x_i - c),
        which has the same energy sum q_i phi_i and the same gradient."""
        n = len(self.q)
        coef = 4 * math.pi / (3 * self.cycle ** 3)
        dip = np.zeros(3)
        for i in range(n):
            dip += (self.x[i] - self.center) * self.q[i]
        if self.dipole_correction == 2:
            self.phi -= coef * ((self.x - self.center) @ dip)
        else:
            dnorm = float(dip @ dip)
            self.phi -= coef * dnorm / n / self.q
        self.grad -= coef * dip[None, :]

    def solve(self, stages="all"):
        """``LaplaceFMM::solve`` (``fmm.cpp:13-81``): the hot block, then the
        dipole correction, the 1/(4 pi) scaling and the re-sort to input order.
        ``stages`` = "all", "near" (P2P only) or "far" (everything but P2P)."""
        if stages in ("all", "far"):
            self.p2m()
            self.m2m()
            self.m2l()
            self.l2l()
            self.l2p()
        if stages in ("all", "near"):
            self.p2p()
        if self.dipole_correction:
            self.dipole_correction_()
        phi, grad = self.phi.copy(), self.grad.copy()
        if self.divide_4pi:
            phi *= INV4PI
            grad *= INV4PI
        out_phi = np.empty_like(phi)
        out_grad = np.empty_like(grad)
        out_phi[self.perm] = phi
        out_grad[self.perm] = grad
        return out_phi, out_grad


    # -- the pass sharded over ranks (test model of rtfmm_b200_shard) ---------
    def shard_owned(self, rank, nranks):
        """The leaves rank `rank` of `nranks` computes (those whose first body
        in tree order lies in [rank n / R, (rank + 1) n / R)) and the cells it
        computes: those leaves' ancestors, and every image cell."""
        c = self.cells
        n = len(self.q)
        parent = [-1] * len(c)
        for i in range(len(c)):
            if c.depth[i] >= 0:
                for k in range(c.cnum[i]):
                    parent[c.coff[i] + k] = i
        leaves = [l for l in self.leaves() if (c.boff[l] * nranks) // max(n, 1) == rank]
        cells = {i for i in range(len(c)) if c.depth[i] < 0}
        for l in leaves:
            a = l
            while a >= 0 and a not in cells:
                cells.add(a)
                a = parent[a]
        return leaves, cells

    def solve_sharded(self, rank, nranks, allreduce):
        """One rank's share of the pass: P2M of its leaves, the exchange
        (`allreduce` sums the leaf q_equiv rows over the ranks in place), M2M
        on the whole tree, M2L / L2L of its cells, L2P and P2P of its leaves.
        Returns (phi, grad) in input order and the mask of the bodies it
        computed (no dipole correction)."""
        leaves, cells = self.shard_owned(rank, nranks)
        self.p2m(leaves=leaves)
        lv = self.leaves()
        buf = np.zeros((len(lv), self.ops.ns))
        own = set(leaves)
        for i, l in enumerate(lv):
            if l in own:
                buf[i] = self.q_equiv[l]
        allreduce(buf)
        for i, l in enumerate(lv):
            self.q_equiv[l] = buf[i]
        self.m2m()
        self.m2l(targets=cells)
        self.l2l(parents=cells)
        self.l2p(leaves=leaves)
        self.p2p(targets=own)
        mask = np.zeros(len(self.q), bool)
        for l in leaves:
            mask[self.cells.boff[l]:self.cells.boff[l] + self.cells.bnum[l]] = True
        phi, grad = self.phi.copy(), self.grad.copy()
        if self.divide_4pi:
            phi *= INV4PI
            grad *= INV4PI
        out_phi = np.empty_like(phi)
        out_grad = np.empty_like(grad)
        out_mask = np.empty_like(mask)
        out_phi[self.perm] = phi
        out_grad[self.perm] = grad
        out_mask[self.perm] = mask
        return out_phi, out_grad, out_mask


def solve(x, q, P, ncrit, images, cycle, **kw):
    return FMM(x, q, P, ncrit, images, cycle, **kw).solve()


# ----------------------------------------------------------------------------
# reference sums and the comparison metric
# ----------------------------------------------------------------------------
def direct_periodic(x, q, images, cycle, targets=None):
    """``LaplaceKernel::direct`` (``kernel.cpp:11-77``): all pairs over
    (3^images)^3 tiles, r = 0 masked.  Returns phi, grad (no 1/4pi)."""
    x = np.asarray(x, dtype=np.float64)
    tgt = np.arange(len(q)) if targets is None else np.asarray(targets)
    dm = (3 ** images - 1) // 2
    phi = np.zeros(len(tgt))
    grad = np.zeros((len(tgt), 3))
    xt = x[tgt]
    for pz in range(-dm, dm + 1):
        for py in range(-dm, dm + 1):
            for px in range(-dm, dm + 1):
                off = np.array([px, py, pz], dtype=np.float64) * cycle
                for c0 in range(0, len(q), 2048):
                    xs = x[c0:c0 + 2048] + off
                    d = xt[:, None, :] - xs[None, :, :]
                    ir = inv_r(d)
                    phi += ir @ q[c0:c0 + 2048]
                    grad -= np.einsum("ts,tsk->tk", (ir ** 3) * q[c0:c0 + 2048][None, :], d)
    return phi, grad


def _ewald_real_pair(xt, xs, qs, alpha, cutoff):
    d = xt[:, None, :] - xs[None, :, :]
    r = np.sqrt(np.sum(d * d, axis=-1))
    m = (r > 0) & (r < cutoff)
    rs = np.where(m, r, 1.0)
    import scipy.special as sp
    e = sp.erfc(alpha * rs)
    pot = np.where(m, e / rs, 0.0) @ qs
    coef = np.where(m, (e + 2 * alpha * rs * np.exp(-alpha * alpha * rs * rs) / math.sqrt(math.pi)) / rs ** 3, 0.0)
    grad = -np.einsum("ts,tsk->tk", coef * qs[None, :], d)
    return pot, grad


def ewald(x, q, cycle, ksize=11, ncrit=64, center=(0.0, 0.0, 0.0), images="reference"):
    """Ewald sum as ``EwaldSolver`` (``3dpp/src/ewald.cpp``) computes it:
    alpha = ksize/L (``ewald.cpp:13``), real part for r < L/2, k-space over
    the (2 ksize + 1)^3 - 1 integer waves (``16-30, 94-109, 177-202``), self
    term -2 alpha q / sqrt(pi) (``112-118``).  Returns phi and grad(phi), in
    input order, no 1/(4 pi) and no dipole term.

    images="reference" restates how the reference picks the periodic image
    of a real-space pair: one offset per pair of leaf cells of its own octree
    (built with ``ncrit``), from the cell centres with a strict |dx| > L/2
    test (``ewald.cpp:121-152``).  Leaf cells exactly L/2 apart therefore
    keep offset 0, and particle pairs that are within the cutoff only through
    the other image are left out.  images="minimum" uses the per-particle
    minimum image instead."""
    x = np.asarray(x, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    n = len(q)
    L = cycle
    alpha = ksize / L
    cutoff = L / 2
    phi = np.zeros(n)
    grad = np.zeros((n, 3))
    if images == "reference":
        cells, perm = build_nonuniform_octree(x, np.asarray(center, dtype=np.float64), L / 2, ncrit)
        xs, qs = x[perm], q[perm]
        leaves = [c for c in range(len(cells)) if cells.is_leaf(c)]
        ph = np.zeros(n)
        gr = np.zeros((n, 3))
        for t in leaves:
            t0, nt = cells.boff[t], cells.bnum[t]
            for s in leaves:
                s0, ns = cells.boff[s], cells.bnum[s]
                dx = cells.x[t] - cells.x[s]
                off = np.where(dx < -L / 2, -L, np.where(dx > L / 2, L, 0.0))
                p_, g_ = _ewald_real_pair(xs[t0:t0 + nt], xs[s0:s0 + ns] + off, qs[s0:s0 + ns], alpha, cutoff)
                ph[t0:t0 + nt] += p_
                gr[t0:t0 + nt] += g_
        phi[perm] = ph
        grad[perm] = gr
    else:
        for c0 in range(0, n, 512):
            xt = x[c0:c0 + 512]
            d = xt[:, None, :] - x[None, :, :]
            d -= L * np.round(d / L)
            r = np.sqrt(np.sum(d * d, axis=-1))
            m = (r > 0) & (r < cutoff)
            rs = np.where(m, r, 1.0)
            import scipy.special as sp
            e = sp.erfc(alpha * rs)
            phi[c0:c0 + 512] += np.where(m, e / rs, 0.0) @ q
            coef = np.where(m, (e + 2 * alpha * rs * np.exp(-alpha * alpha * rs * rs) / math.sqrt(math.pi)) / rs ** 3, 0.0)
            grad[c0:c0 + 512] -= np.einsum("ts,tsk->tk", coef * q[None, :], d)
    kr = np.arange(-ksize, ksize + 1)
    K = np.stack(np.meshgrid(kr, kr, kr, indexing="ij"), axis=-1).reshape(-1, 3)
    K = K[np.any(K != 0, axis=1)].astype(np.float64)
    scale = 2 * math.pi / L
    coef = 4 * math.pi / L ** 3
    for w0 in range(0, len(K), 512):
        kw = K[w0:w0 + 512]
        ph_s = (x @ kw.T) * scale
        S = (q[:, None] * np.exp(-1j * ph_s)).sum(axis=0)
        k2 = np.sum(kw * kw, axis=1) * scale * scale
        S *= coef * np.exp(-k2 / (4 * alpha * alpha)) / k2
        e = np.exp(1j * ph_s) * S[None, :]
        phi += e.real.sum(axis=1)
        grad += (np.real(e * 1j) * scale) @ kw
    phi -= (2 / math.sqrt(math.pi)) * q * alpha
    return phi, grad


def compare(p1, f1, q1, p2, f2, q2):
    """``compare`` (``3dpp/src/body.cpp:131-175``); the second set is the norm."""
    pdif = np.sum((p1 - p2) ** 2)
    pnrm = np.sum(p2 ** 2)
    fdif = np.sum((f1 - f2) ** 2)
    fnrm = np.sum(f2 ** 2)
    e1 = float(np.sum(p1 * q1))
    e2 = float(np.sum(p2 * q2))
    n = len(p1)
    return {"l2p": math.sqrt(pdif / pnrm), "l2f": math.sqrt(fdif / fnrm),
            "l2e": math.sqrt((e1 - e2) ** 2 / e2 / e2),
            "rmsp": math.sqrt(pdif / n), "rmsf": math.sqrt(fdif / n),
            "energy1": e1, "energy2": e2}
