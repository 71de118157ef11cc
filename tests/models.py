"""Model builders shared by the parity tests, the golden-vector generator and
the benchmark.

Every builder takes the Radia-compatible module to build with -- the
reference ``radia`` module (compiled under oracle/_ref) or this repository's
``radiacuda_b200.rad`` -- and uses only API calls both provide, so the same
seeded model is built on both sides of a parity comparison.  Inputs are
seeded synthetic geometries with the shapes of the workloads the hot path is
measured on (magnet arrays, iron yokes with coils, tetrahedral meshes,
undulators).
"""
from __future__ import annotations

import numpy as np

TET_FACES = [[1, 2, 3], [1, 4, 2], [2, 4, 3], [3, 4, 1]]
CUBE = [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]]
KUHN = [[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6], [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]]


def reset(R):
    R.UtiDelAll()
    R.FldLenRndSw("off")


# ---------------------------------------------------------------------------
# permanent-magnet array: 16 blocks 10 mm on a 4x4 grid, anisotropic MatLin,
# each subdivided 3x3x3 -> 432 cuboids (the small linear workload)
# ---------------------------------------------------------------------------
def magnet_array(R, nside=4, div=3, seed=12345):
    reset(R)
    rng = np.random.default_rng(seed)
    blocks = []
    for i in range(nside):
        for j in range(nside):
            v = rng.normal(size=3)
            mr = (1.2 * v / np.linalg.norm(v)).tolist()
            c = [-18.0 + 12.0 * i, -18.0 + 12.0 * j, 0.0]
            b = R.ObjRecMag(c, [10, 10, 10], mr)
            R.MatApl(b, R.MatLin([0.06, 0.17], mr))
            if div > 1:
                R.ObjDivMag(b, [div, div, div])
            blocks.append(b)
    return R.ObjCnt(blocks)


def magnet_array_points(nxy=25, nz=16):
    x = np.linspace(-23, 23, nxy) + 0.1371
    z = np.linspace(10, 25, nz) + 0.0517
    X, Y, Z = np.meshgrid(x, x, z, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


# ---------------------------------------------------------------------------
# symmetric magnets: mirrored / rotated cuboids (image handling)
# ---------------------------------------------------------------------------
def sym_blocks(R, div=2):
    reset(R)
    a = R.ObjRecMag([12, 7, 4], [10, 6, 5], [0.3, 1.0, 0.2])
    R.MatApl(a, R.MatLin([0.05, 0.15], [0.3, 1.0, 0.2]))
    # centres kept off the other blocks' face planes: with FldLenRndSw('off')
    # the reference returns NaN for observation points on a face plane
    b = R.ObjRecMag([30, 5.3, 9.1], [6, 8, 7], [-0.4, 0.2, 0.9])
    R.MatApl(b, R.MatLin([0.06, 0.12], [-0.4, 0.2, 0.9]))
    R.ObjDivMag(a, [div, div, 1])
    R.ObjDivMag(b, [1, div, div])
    g = R.ObjCnt([a, b])
    R.TrfZerPerp(g, [0, 0, 0], [1, 0, 0])
    R.TrfZerPara(g, [0, 0, 0], [0, 0, 1])
    c = R.ObjRecMag([0, 40, 0], [8, 8, 8], [0.0, 0.0, 1.1])
    R.MatApl(c, R.MatLin([0.06, 0.17], [0.0, 0.0, 1.1]))
    rot = R.TrfRot([0, 40, 0], [1, 1, 0], 0.7)
    R.TrfOrnt(c, rot)
    return R.ObjCnt([g, c])


# ---------------------------------------------------------------------------
# iron dipole: saturating yoke (MatSatIsoFrm) from cuboids, two mirror planes
# (4 images per element) and a racetrack coil placed without symmetry
# ---------------------------------------------------------------------------
def iron_dipole(R, n_target=4000, gap=40.0, coil=True, ni=10000.0):
    """C-shaped yoke in the quadrant x>=0, z>=0 (mirrored to the full magnet)."""
    reset(R)
    hg = 0.5 * gap
    # (x, y = depth, z): pole above the gap, top bar, return leg
    pole = ([15.0, 0.0, hg + 20.0], [30.0, 80.0, 40.0])
    top = ([50.0, 0.0, hg + 55.0], [100.0, 80.0, 30.0])
    leg = ([85.0, 0.0, 0.5 * (hg + 40.0)], [30.0, 80.0, hg + 40.0])
    parts = [pole, top, leg]
    vol = sum(d[0] * d[1] * d[2] for _, d in parts)
    h = (vol / n_target) ** (1.0 / 3.0)
    ids = []
    for c, d in parts:
        b = R.ObjRecMag(c, d, [0, 0, 0])
        k = [max(1, int(round(x / h))) for x in d]
        if k != [1, 1, 1]:
            R.ObjDivMag(b, k)
        ids.append(b)
    yoke = R.ObjCnt(ids)
    R.MatApl(yoke, R.MatSatIsoFrm([20000, 2], [0.1, 2], [0.1, 2]))
    R.TrfZerPerp(yoke, [0, 0, 0], [1, 0, 0])
    R.TrfZerPara(yoke, [0, 0, 0], [0, 0, 1])
    if not coil:
        return R.ObjCnt([yoke])
    rmin, rmax, hc = 2.0, 22.0, 30.0
    j = ni / (hc * (rmax - rmin))
    c = R.ObjRaceTrk([0, 0, hg + 20.0], [rmin, rmax], [60.0, 80.0], hc, 6, j, "man", "z")
    return R.ObjCnt([yoke, c])


def iron_dipole_points(n=100, gap=40.0):
    x = np.linspace(-45, 45, n) + 0.1371
    y = np.linspace(-45, 45, n) + 0.0913
    z = np.linspace(-0.45 * gap, 0.45 * gap, n) + 0.0517
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


# ---------------------------------------------------------------------------
# tetrahedral mesh: jittered Kuhn lattice with slivers, linear iso chi
# ---------------------------------------------------------------------------
def tet_mesh_vertices(ncell=15, n_tets=20000, edge=2.0, seed=2024, sliver_frac=0.02):
    rng = np.random.default_rng(seed)
    g = ncell + 1
    idx = np.arange(g ** 3).reshape(g, g, g)
    P = np.stack(np.meshgrid(np.arange(g), np.arange(g), np.arange(g), indexing="ij"), axis=-1).reshape(-1, 3).astype(float)
    P = P * edge + rng.uniform(-0.02, 0.02, size=P.shape) * edge
    tets = []
    for i in range(ncell):
        for j in range(ncell):
            for k in range(ncell):
                corner = [idx[i + c[0], j + c[1], k + c[2]] for c in CUBE]
                for t in KUHN:
                    tets.append([corner[q] for q in t])
    tets = tets[:n_tets]
    V = [P[t].copy() for t in tets]
    ns = int(round(sliver_frac * len(V)))
    pick = rng.choice(len(V), size=ns, replace=False)
    for s in pick:
        v = V[s]
        # move the 4th vertex toward the opposite face (aspect up to ~50)
        c = v[:3].mean(axis=0)
        v[3] = c + (v[3] - c) * rng.uniform(0.02, 0.2)
    return V


def tet_mesh(R, ncell=15, n_tets=20000, chi=1000.0, bext=(0, 0, 1), seed=2024):
    reset(R)
    V = tet_mesh_vertices(ncell, n_tets, seed=seed)
    ids = [R.ObjPolyhdr(v.tolist(), TET_FACES) for v in V]
    body = R.ObjCnt(ids)
    R.MatApl(body, R.MatLin([chi, chi], [0, 0, 1e-12]))
    bk = R.ObjBckg(list(bext))
    return R.ObjCnt([body, bk]), body


def tet_mesh_points(n=1_000_000, ncell=15, edge=2.0, margin=2.0, seed=7):
    """Random points outside the body's bounding box + margin."""
    rng = np.random.default_rng(seed)
    L = ncell * edge
    lo, hi = -margin - 0.25 * L, L + margin + 0.25 * L
    out = np.empty((0, 3))
    while out.shape[0] < n:
        p = rng.uniform(lo, hi, size=(2 * n, 3))
        inside = np.all((p > -margin) & (p < L + margin), axis=1)
        out = np.concatenate([out, p[~inside]], axis=0)
    return out[:n]


# ---------------------------------------------------------------------------
# planar undulator (shimming workload)
# ---------------------------------------------------------------------------
def undulator(R, nper_row=40, div=2, seed_m=4, seed_a=5, period=20.0, gap=10.0,
              mr_offsets=None, c_offsets=None):
    """2 rows of blocks 50x10x5 mm (x,y,z), 4 blocks per period along z,
    M rotating 90 deg per block.  Returns (model, block handles)."""
    reset(R)
    rm = np.random.default_rng(seed_m)
    ra = np.random.default_rng(seed_a)
    nb = 2 * nper_row
    mag = 1.3 * (1.0 + 0.02 * rm.uniform(-1, 1, nb))
    tilt = np.deg2rad(1.0) * ra.uniform(0, 1, nb)
    az = ra.uniform(0, 2 * np.pi, nb)
    blocks = []
    zlen = 5.0
    for row in range(2):
        y = (0.5 * gap + 5.0) * (1 if row == 0 else -1)
        for k in range(nper_row):
            b = row * nper_row + k
            z = (k - 0.5 * (nper_row - 1)) * zlen
            dirs = [(0, 1, 0), (0, 0, 1), (0, -1, 0), (0, 0, -1)]
            d = np.array(dirs[k % 4], float) * (1 if row == 0 else -1) if k % 2 == 0 else np.array(dirs[k % 4], float)
            # tilt by up to 1 degree
            perp = np.cross(d, [1.0, 0.0, 0.0])
            perp = perp / np.linalg.norm(perp)
            perp2 = np.cross(d, perp)
            dt = d * np.cos(tilt[b]) + np.sin(tilt[b]) * (np.cos(az[b]) * perp + np.sin(az[b]) * perp2)
            mr = mag[b] * dt
            if mr_offsets is not None:
                mr = mr + mr_offsets[b]
            c = np.array([0.0, y, z])
            if c_offsets is not None:
                c = c + c_offsets[b]
            h = R.ObjRecMag(c.tolist(), [50, 10, 5], mr.tolist())
            R.MatApl(h, R.MatLin([0.05, 0.15], mr.tolist()))
            if div > 1:
                R.ObjDivMag(h, [div, div, div])
            blocks.append(h)
    return R.ObjCnt(blocks), blocks


def undulator_points(n=4000, nper_row=40):
    zspan = nper_row * 5.0
    z = np.linspace(-0.5 * zspan, 0.5 * zspan, n) + 0.0517
    return np.stack([np.full(n, 0.1371), np.full(n, 0.0913), z], axis=1)


# ---------------------------------------------------------------------------
# hybrid undulator: NdFeB blocks (magnetized along +-z) alternating with
# saturating iron poles along z, upper half modelled, the lower half by the
# mirror plane y = 0 (2 images per element)
# ---------------------------------------------------------------------------
HYB_POLE = (40.0, 20.0, 4.0)    # x, y, z widths of a pole
HYB_BLOCK = (50.0, 25.0, 6.0)   # of a block; period = 2 (pole + block) = 20 mm


def hybrid_undulator(R, n_pairs=80, pole_div=(4, 4, 4), block_div=(2, 2, 3), gap=10.0, mr=1.25, seed=6,
                     pole_dz=None, block_mr=None):
    """n_pairs blocks alternating with n_pairs poles.  pole_dz[k] changes the
    z width of pole k (centre fixed); block_mr[k] replaces block k's remanence
    vector.  Returns (model, pole handles, block handles, pole centres)."""
    reset(R)
    rng = np.random.default_rng(seed)
    pz, bz = HYB_POLE[2], HYB_BLOCK[2]
    step = pz + bz
    z0 = -0.5 * n_pairs * step
    poles, blocks, pc = [], [], []
    for k in range(n_pairs):
        zp = z0 + k * step + 0.5 * pz
        zb = zp + 0.5 * (pz + bz)
        dz = pz + (0.0 if pole_dz is None else pole_dz[k])
        p = R.ObjRecMag([0.0, 0.5 * gap + 0.5 * HYB_POLE[1], zp], [HYB_POLE[0], HYB_POLE[1], dz], [0, 0, 0])
        if pole_div != (1, 1, 1):
            R.ObjDivMag(p, list(pole_div))
        poles.append(p)
        pc.append([0.0, 0.5 * gap + 0.5 * HYB_POLE[1], zp])
        if block_mr is not None:
            m = np.asarray(block_mr[k], float)
        else:
            m = np.array([0.0, 0.0, mr * (1 if k % 2 == 0 else -1)]) * (1.0 + 0.01 * rng.uniform(-1, 1))
        b = R.ObjRecMag([0.0, 0.5 * gap + 0.5 + 0.5 * HYB_BLOCK[1], zb], list(HYB_BLOCK), m.tolist())
        R.MatApl(b, R.MatLin([0.05, 0.15], m.tolist()))
        if block_div != (1, 1, 1):
            R.ObjDivMag(b, list(block_div))
        blocks.append(b)
    gp = R.ObjCnt(poles)
    R.MatApl(gp, R.MatSatIsoFrm([2000, 1.5], [100, 0.4], [10, 0.2]))
    g = R.ObjCnt([gp] + blocks)
    R.TrfZerPara(g, [0, 0, 0], [0, 1, 0])
    return g, poles, blocks, np.array(pc)


def hybrid_points(n=100_000, n_pairs=80, seed=9):
    """Points in the gap over the length of the device (off every face plane)."""
    rng = np.random.default_rng(seed)
    L = n_pairs * (HYB_POLE[2] + HYB_BLOCK[2])
    return np.stack([rng.uniform(-15, 15, n) + 0.0137, rng.uniform(-4, 4, n) + 0.0071,
                     rng.uniform(-0.5 * L, 0.5 * L, n) + 0.0517], axis=1)


# ---------------------------------------------------------------------------
# small models for the adjoint tests: linear anisotropic blocks with images,
# a rotated block, a coil and a background field; and a small hybrid
# ---------------------------------------------------------------------------
def adjoint_linear(R):
    g = sym_blocks(R, div=2)
    coil = R.ObjRaceTrk([20.0, 20.0, 25.0], [3, 9], [10, 14], 6, 4, 2.0, "man", "z")
    bk = R.ObjBckg([0.05, -0.02, 0.1])
    return R.ObjCnt([g, coil, bk])


def adjoint_points(n=160, seed=31):
    rng = np.random.default_rng(seed)
    return rng.uniform([-45, -15, -25], [45, 55, 25], size=(n, 3)) + np.array([0.0137, 0.0071, 0.0053])


# ---------------------------------------------------------------------------
# mixed cuboids + tetrahedra with a symmetry, saturating material and a coil
# ---------------------------------------------------------------------------
def mixed_sym(R, seed=3):
    reset(R)
    rng = np.random.default_rng(seed)
    tets = []
    for _ in range(12):
        base = rng.uniform([40, 5, 8], [70, 30, 30])
        v = base + rng.uniform(2, 8, size=(4, 3))
        tets.append(R.ObjPolyhdr(v.tolist(), TET_FACES))
    ga = R.ObjCnt(tets)
    recs = []
    for i in range(3):
        recs.append(R.ObjRecMag([10.0 + 9 * i, 12.0, 6.0], [8.0, 6.0, 5.0], [0, 0, 0]))
    gb = R.ObjCnt(recs)
    R.ObjDivMag(gb, [2, 1, 2])
    mat = R.MatSatIsoFrm([2000, 1.5], [100, 0.4], [10, 0.2])
    R.MatApl(ga, mat)
    R.MatApl(gb, mat)
    R.TrfZerPerp(ga, [0, 0, 0], [0, 1, 0])
    R.TrfZerPara(gb, [0, 0, 0], [0, 0, 1])
    coil = R.ObjRaceTrk([0, 0, 40], [60, 80], [10, 20], 15, 8, 2.0, "man", "z")
    arc = R.ObjArcCur([20, -30, -20], [5, 9], [0.3, 2.9], 6, 10, 3.0, "man", "x")
    return R.ObjCnt([ga, gb, coil, arc])


# ---------------------------------------------------------------------------
# extruded polygons along x, y and z, anisotropic linear and saturating
# materials (with FldLenRndSw('off') the reference keeps even the rectangle
# as an extruded polygon)
# ---------------------------------------------------------------------------
def thckpgn_model(R):
    reset(R)
    hexagon = [[6.0 * np.cos(k * np.pi / 3) + 0.3, 6.0 * np.sin(k * np.pi / 3) - 0.2] for k in range(6)]
    a = R.ObjThckPgn(4.0, 8.0, hexagon, "x", [0.9, 0.2, -0.1])
    b = R.ObjThckPgn(20.0, 5.0, [[0.0, 0.0], [9.0, 1.5], [3.0, 7.0]], "y", [0.1, 1.1, 0.3])
    pent = [[5.0 * np.cos(2 * np.pi * k / 5) + 25.0, 5.0 * np.sin(2 * np.pi * k / 5) - 3.0] for k in range(5)]
    c = R.ObjThckPgn(-7.0, 6.0, pent, "z", [0.0, 0.0, 1.0])
    d = R.ObjThckPgn(12.0, 4.0, [[30.0, 10.0], [38.0, 10.0], [38.0, 16.0], [30.0, 16.0]], "z", [0.5, 0.0, 0.0])
    R.MatApl(a, R.MatLin([0.05, 0.15], [0.9, 0.2, -0.1]))
    R.MatApl(b, R.MatLin([0.06, 0.12], [0.1, 1.1, 0.3]))
    R.MatApl(c, R.MatSatIsoFrm([2000, 1.5], [100, 0.4], [10, 0.2]))
    R.MatApl(d, R.MatLin([0.05, 0.15], [0.5, 0.0, 0.0]))
    return R.ObjCnt([a, b, c, d])


# ---------------------------------------------------------------------------
# the reference's MPI-solve regression models (tests/test_mpi_solve.py of the
# reference), rebuilt with the same seeded draws so the golden B values of
# its tests/_mpi_solve_reference.json apply
# ---------------------------------------------------------------------------
def mpi_solve_model(R, kind="small"):
    R.UtiDelAll()
    R.FldLenRndSw("on")   # the golden values were made with the default setting
    rng = np.random.default_rng(11)
    ids = []
    if kind == "large":
        for _ in range(1100):
            c = rng.uniform([-80, -80, -40], [80, 80, 40]).tolist()
            d = rng.uniform(2.0, 4.0, 3).tolist()
            ids.append(R.ObjRecMag(c, d))
        body = R.ObjCnt(ids)
    else:
        for _ in range(60):
            base = rng.uniform([20, 5, 5], [90, 40, 40])
            v = base + rng.uniform(2, 10, size=(4, 3))
            ids.append(R.ObjPolyhdr(v.tolist(), TET_FACES))
        if kind == "mixed":
            for i in range(3):
                for j in range(2):
                    for k in range(2):
                        ids.append(R.ObjRecMag([30.0 + i * 12, 10.0 + j * 11, 8.0 + k * 9], [10.0, 8.0, 7.0]))
        body = R.ObjCnt(ids)
        R.TrfZerPerp(body, [0, 0, 0], [1, 0, 0])
        R.TrfZerPara(body, [0, 0, 0], [0, 0, 1])
    R.MatApl(body, R.MatSatIsoFrm([20000, 2], [0.1, 2], [0.1, 2]))
    coil = R.ObjRaceTrk([0, 0, 30], [70, 90], [0, 0], 15, 10, 3.0, "man", "z")
    return R.ObjCnt([body, coil])


MPI_SOLVE_POINTS = [[25.0, 10.0, 0.0], [60.0, 30.0, 5.0]]
