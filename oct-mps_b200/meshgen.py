"""Synthetic OCT-MPS inputs in the reference's file formats.

The benchmark geometries are boxes of turbid tissue with ellipsoidal
inclusions, meshed as a structured grid of cubes each split into the six
Kuhn (Freudenthal) tetrahedra along its main diagonal, which makes a
conforming mesh.  A tet's region is decided by its centroid.  Rules that
keep the reference's own code usable on these meshes:

* The z = 0 layer (the probe's surface) is emitted first, so that the
  reference's root search (src/mesh.cpp:263, a loop over tets in file order)
  meets the root early.
* The grid is shifted so that every probe position lies strictly inside a
  top-face triangle: off the x and y grid lines and off the cube diagonal
  that splits each top square (FindRootofGraph, src/mesh.cpp:276-283, needs
  the probe on exactly one face plane of the root tet).
* Vertices are written with 9 significant digits; the reader parses them
  as float (src/mesh.cpp:136-143).

Units are the reference's: cm and 1/cm.  Writers follow the .opt
(src/octmps_io.cpp:504-645), .mci (src/bias.cpp:9-110) and .mesh
(src/mesh.cpp:103-158) layouts.
"""
import os

import numpy as np

# Kuhn split of the unit cube: tet k visits the cube's corners along the
# axis permutation PERMS[k], from (0,0,0) to (1,1,1).
PERMS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


class Inclusion:
    """Ellipsoid (x-cx)^2/ax^2 + (y-cy)^2/ay^2 + (z-cz)^2/az^2 <= 1 of one region."""

    def __init__(self, center, semi_axes, region):
        self.c = np.asarray(center, float)
        self.a = np.asarray(semi_axes, float)
        self.region = region

    def inside(self, p):
        return np.sum(((p - self.c) / self.a) ** 2, axis=-1) <= 1.0


def grid_mesh(nx, ny, nz, h, x0, y0, inclusions, background=1):
    """Vertices (N,3) and tets (T,5: four 1-based vertex ids + region)."""
    xs = x0 + h * np.arange(nx + 1)
    ys = y0 + h * np.arange(ny + 1)
    zs = h * np.arange(nz + 1)
    vid = lambda i, j, k: (k * (ny + 1) + j) * (nx + 1) + i  # noqa: E731
    K, J, I = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    verts = np.stack([xs[I.ravel()], ys[J.ravel()], zs[K.ravel()]], axis=1)
    # cubes in z-major, then y, then x order
    ck, cj, ci = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ck, cj, ci = ck.ravel(), cj.ravel(), ci.ravel()
    tets = np.zeros((len(ck), 6, 5), np.int64)
    for t, perm in enumerate(PERMS):
        off = np.zeros(3, int)
        corners = [vid(ci, cj, ck)]
        for ax in perm:
            off[ax] += 1
            corners.append(vid(ci + off[0], cj + off[1], ck + off[2]))
        tets[:, t, :4] = np.stack(corners, axis=1) + 1
    tets = tets.reshape(-1, 5)
    cent = verts[tets[:, :4] - 1].mean(axis=1)
    region = np.full(len(tets), background, np.int64)
    for inc in inclusions:
        region[inc.inside(cent)] = inc.region
    tets[:, 4] = region
    return verts, tets


def write_mesh(path, verts, tets):
    with open(path, "w") as f:
        f.write(f"{len(verts)}\n{len(tets)}\n")
        np.savetxt(f, verts, fmt="%.9g %.9g %.9g")
        np.savetxt(f, tets, fmt="%d %d %d %d %d")


def write_opt(path, n_photons, regions, probe, ambient_n=1.0, name="sample.mco"):
    """regions: list of (n, mua, mus, g) for regions 1..R; probe: (start, step, end)."""
    with open(path, "w") as f:
        f.write("# OCT-MPS input (generated)\n")
        f.write("1.0\t\t# file version\n1\t\t# number of runs\n\n")
        f.write(f"{name}\tA\t\t# output file name, ASCII\n")
        f.write(f"{int(n_photons)}\t\t# No. of photons\n\n")
        f.write(f"{len(regions)}\t\t# Number of regions\n")
        f.write("#n\tmua\tmus\tg\n")
        f.write(f"{ambient_n!r}\t\t# n for ambient medium\n")
        for k, (n, mua, mus, g) in enumerate(regions, 1):
            f.write(f"{n!r}\t{mua!r}\t{mus!r}\t{g!r}\t# region {k}\n")
        f.write("\n#Start\tStep\tEnd\n")
        f.write(f"{probe[0]!r}\t{probe[1]!r}\t{probe[2]!r}\n")


def write_mci(path, type_bias=37, bias_a=0.925, depth_min=0.0, depth_max=0.15, lc=0.0015,
              radius=0.001, angle_deg=5.0, p_bias=0.5, maxrel=0.01, type_simulation=1,
              record=0):
    with open(path, "w") as f:
        f.write("####\n# BiasStartup.mci (generated)\n####\n")
        for v, c in [(type_simulation, "Type of Simulation"), (type_bias, "Type of Bias"),
                     (bias_a, "Backward bias coefficient"), (depth_min, "Target depth min [cm]"),
                     (depth_max, "Target depth max [cm]"), (lc, "Coherence length source [cm]"),
                     (record, "Record photons flag"), (radius, "Max collecting radius [cm]"),
                     (angle_deg, "Max collecting angle [deg]"), (p_bias, "Probability additional bias"),
                     (maxrel, "Max rel. contrib. to bin")]:
            f.write(f"{v!r}\t\t# {c}\n")


TISSUE = (1.33, 0.15, 60.0, 0.9)  # n, mua [1/cm], mus [1/cm], g


def config_plain_ascan(out_dir, n_photons=100_000, nx=40, ny=40, nz=30):
    """Config 1: 2 x 2 x 1.5 mm box, sphere r = 0.3 mm at depth 0.6 mm,
    40x40x30 cubes (288,000 tets), one A-scan at x = 0, 1e5 packets."""
    h = 0.2 / nx
    x0 = -0.1 - 0.02 * h
    y0 = -0.1 - 0.51 * h
    incl = [Inclusion((0.0, 0.0, 0.06), (0.03, 0.03, 0.03), 2)]
    verts, tets = grid_mesh(nx, ny, nz, h, x0, y0, incl)
    return _write_deck(out_dir, "plain", verts, tets, n_photons,
                       [TISSUE, (1.40, 0.2, 90.0, 0.9)], (0.0, 0.001, 0.0005))


def config_bscan(out_dir, n_ascans=256, n_photons=1_000_000, nx=64, ny=32, nz=31):
    """Config 2: 4 x 2 x 2 mm box with an ellipsoid (semi-axes 1.2/0.6/0.3 mm,
    depth 0.7 mm) and two spheres (r = 0.2 mm, depths 0.5 and 0.9 mm),
    64x32x31 cubes of 62.5 um (380,928 tets), A-scans every 10 um."""
    h = 0.4 / nx
    x0 = -0.2 - 0.02 * h
    y0 = -0.1 - 0.51 * h
    incl = [Inclusion((0.0, 0.0, 0.07), (0.12, 0.06, 0.03), 2),
            Inclusion((-0.06, 0.0, 0.05), (0.02, 0.02, 0.02), 3),
            Inclusion((0.06, 0.0, 0.09), (0.02, 0.02, 0.02), 3)]
    verts, tets = grid_mesh(nx, ny, nz, h, x0, y0, incl)
    start = -0.001 * (n_ascans // 2)
    probe = (start, 0.001, start + 0.001 * n_ascans - 0.0005)
    return _write_deck(out_dir, "bscan", verts, tets, n_photons,
                       [TISSUE, (1.40, 0.15, 90.0, 0.9), (1.38, 0.3, 120.0, 0.95)], probe)


def layered_grid(nx, ny, h, x0, y0, surfaces, cells_per_layer):
    """A structured grid whose node z follows the layer surfaces: column
    (i, j) runs from surface 0 down through each layer, with
    cells_per_layer[l] cells spaced evenly between surfaces l and l+1, so every
    interface is a face of the grid.  surfaces[l](X, Y) gives depth.  Regions
    are the layer numbers (1-based)."""
    nz = int(sum(cells_per_layer))
    xs = x0 + h * np.arange(nx + 1)
    ys = y0 + h * np.arange(ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="xy")  # [ny+1, nx+1]
    Z = np.zeros((nz + 1, ny + 1, nx + 1))
    layer_of_cell = np.zeros(nz, np.int64)
    k = 0
    for l, n in enumerate(cells_per_layer):
        top, bot = surfaces[l](X, Y), surfaces[l + 1](X, Y)
        for c in range(n):
            Z[k + c] = top + (bot - top) * (c / n)
            layer_of_cell[k + c] = l + 1
        k += n
    Z[nz] = surfaces[-1](X, Y)
    verts = np.stack([np.broadcast_to(X, Z.shape).ravel(), np.broadcast_to(Y, Z.shape).ravel(),
                      Z.ravel()], axis=1)
    vid = lambda i, j, kk: (kk * (ny + 1) + j) * (nx + 1) + i  # noqa: E731
    ck, cj, ci = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ck, cj, ci = ck.ravel(), cj.ravel(), ci.ravel()
    tets = np.zeros((len(ck), 6, 5), np.int64)
    for t, perm in enumerate(PERMS):
        off = np.zeros(3, int)
        corners = [vid(ci, cj, ck)]
        for ax in perm:
            off[ax] += 1
            corners.append(vid(ci + off[0], cj + off[1], ck + off[2]))
        tets[:, t, :4] = np.stack(corners, axis=1) + 1
        tets[:, t, 4] = layer_of_cell[ck]
    return verts, tets.reshape(-1, 5)


def config_layers(out_dir, n_photons=10_000_000, nx=60, ny=60, nz=46, n_ascans=64):
    """Config 3, the precision study: a 2 x 2 x 1.5 mm slab of four layers
    (0.1 / 0.2 / 0.4 / 0.8 mm; mu_s 4 / 10 / 7 / 9 per mm; g 0.9 / 0.95 / 0.9 /
    0.85; n 1.33 / 1.40 / 1.37 / 1.35; mu_a 0.01 / 0.02 / 0.03 / 0.02 per mm)
    whose two middle interfaces are tilted 5 degrees about y.  60x60x46 mapped
    cells (993,600 tets), about 1 um depth bins (Lc = 6 um), 64 A-scans 10 um
    apart."""
    h = 0.2 / nx
    x0 = -0.1 - 0.02 * h
    y0 = -0.1 - 0.51 * h
    tilt = np.tan(np.radians(5.0))
    surfaces = [lambda X, Y: 0.0 * X, lambda X, Y: 0.01 + 0.0 * X,
                lambda X, Y: 0.03 + tilt * X, lambda X, Y: 0.07 + tilt * X,
                lambda X, Y: 0.15 + 0.0 * X]
    thick = np.array([0.01, 0.02, 0.04, 0.08])
    cells = np.maximum(1, np.round(thick / thick.sum() * nz)).astype(int)
    cells[-1] += nz - cells.sum()
    verts, tets = layered_grid(nx, ny, h, x0, y0, surfaces, cells)
    regions = [(1.33, 0.1, 40.0, 0.9), (1.40, 0.2, 100.0, 0.95), (1.37, 0.3, 70.0, 0.9),
               (1.35, 0.2, 90.0, 0.85)]
    start = -0.001 * (n_ascans // 2)
    probe = (start, 0.001, start + 0.001 * n_ascans - 0.0005)
    return _write_deck(out_dir, "layers", verts, tets, n_photons, regions, probe, lc=0.0006)


def config_random_job(out_dir, rng, index, target_tets=None, n_photons=None):
    """Config 4, one job of the batched uneven set: the 2 x 2 x 1.5 mm box
    with 1-4 ellipsoid inclusions (semi-axes 0.1-0.8 mm, mu_s 5-15 per mm, g
    0.8-0.95, n 1.33-1.45), a grid sized for 50k-800k tets and a log-uniform
    number of packets in 1e4-1e7."""
    tets = target_tets or int(10 ** rng.uniform(np.log10(5e4), np.log10(8e5)))
    n = max(4, int(round((tets / (6 * 0.75)) ** (1 / 3))))
    nx, ny, nz = n, n, max(3, int(round(0.75 * n)))
    h = 0.2 / nx
    x0 = -0.1 - 0.02 * h
    y0 = -0.1 - 0.51 * h
    regions = [TISSUE]
    incl = []
    for _ in range(int(rng.integers(1, 5))):
        a = rng.uniform(0.01, 0.08, 3)
        c = (rng.uniform(-0.06, 0.06), rng.uniform(-0.06, 0.06), rng.uniform(0.03, 0.12))
        regions.append((float(rng.uniform(1.33, 1.45)), 0.15, float(rng.uniform(50, 150)),
                        float(rng.uniform(0.8, 0.95))))
        incl.append(Inclusion(c, a, len(regions)))
    verts, tets_arr = grid_mesh(nx, ny, nz, h, x0, y0, incl)
    photons = n_photons or int(10 ** rng.uniform(4, 7))
    return _write_deck(out_dir, f"job{index}", verts, tets_arr, photons, regions,
                       (0.0, 0.001, 0.0005))


def config_small(out_dir, n_photons=20_000, nx=8, ny=8, nz=6, matched=False):
    """A small deck of the same construction for quick parity checks."""
    h = 0.2 / nx
    x0 = -0.1 - 0.02 * h
    y0 = -0.1 - 0.51 * h
    incl = [Inclusion((0.0, 0.0, 0.06), (0.05, 0.05, 0.04), 2)]
    verts, tets = grid_mesh(nx, ny, nz, h, x0, y0, incl)
    regions = [(1.0, 1.5, 60.0, 0.9), (1.0, 3.0, 120.0, 0.9)] if matched else \
        [TISSUE, (1.40, 0.2, 90.0, 0.9)]
    return _write_deck(out_dir, "small", verts, tets, n_photons, regions, (0.0, 0.001, 0.0005))


def _write_deck(out_dir, stem, verts, tets, n_photons, regions, probe, **mci):
    os.makedirs(out_dir, exist_ok=True)
    paths = {k: os.path.join(out_dir, f"{stem}.{k}") for k in ("mesh", "opt", "mci")}
    write_mesh(paths["mesh"], verts, tets)
    write_opt(paths["opt"], n_photons, regions, probe)
    write_mci(paths["mci"], **mci)
    paths["n_tets"] = len(tets)
    return paths
