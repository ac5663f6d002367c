"""Seeded synthetic page scenes shared by the CPU and GPU page tests."""

import numpy as np


def box_occupancy(shape, rng=None, blobs=0):
    """Blocked u8 field of a box window: the one-cell halo plus seeded blobs."""
    sx, sy, sz = shape
    occ = np.zeros((sz, sy, sx), np.uint8)
    occ[0, :, :] = occ[-1, :, :] = 1
    occ[:, 0, :] = occ[:, -1, :] = 1
    occ[:, :, 0] = occ[:, :, -1] = 1
    if rng is not None:
        zz, yy, xx = np.mgrid[0:sz, 0:sy, 0:sx]
        for _ in range(blobs):
            c = rng.uniform([2, 2, 2], [sx - 2, sy - 2, sz - 2])
            r = rng.uniform(2, 5, size=3)
            occ |= ((((xx - c[0]) / r[0]) ** 2 + ((yy - c[1]) / r[1]) ** 2 + ((zz - c[2]) / r[2]) ** 2) < 1)
    return occ.reshape(-1)


def blob_kernel(shape, rng):
    kx, ky, kz = shape
    zz, yy, xx = np.mgrid[0:kz, 0:ky, 0:kx]
    c = (np.array([kx, ky, kz]) - 1) / 2
    r = np.array([kx, ky, kz]) / 2
    d = ((xx - c[0]) / r[0]) ** 2 + ((yy - c[1]) / r[1]) ** 2 + ((zz - c[2]) / r[2]) ** 2
    k = (d + rng.normal(0, 0.15, d.shape) < 1.0).astype(np.uint8)
    k[kz // 2, ky // 2, kx // 2] = 1
    return k.reshape(-1)


def scene(seed, shape=(40, 36, 30), kernel_shape=(9, 7, 8), blobs=6, cuboid=False):
    rng = np.random.default_rng(seed)
    env_first = (-1, -1, -1)
    occ = box_occupancy(shape, rng, blobs)
    if cuboid:
        ker = np.ones(int(np.prod(kernel_shape)), np.uint8)
    else:
        ker = blob_kernel(kernel_shape, rng)
    kernel_first = tuple(int(v) for v in rng.integers(-4, 1, size=3))
    lattice = (0.0, 0.0, 0.0, 1.0)
    height = float(shape[2] - 2)
    max_z = float(kernel_shape[2]) / 2
    return dict(env_first=env_first, env_shape=shape, occ=occ, kernel_first=kernel_first,
                kernel_shape=kernel_shape, kernel=ker, lattice=lattice, max_z=max_z, cmin_z=0.0, height=height)
