"""Structured block meshes in mesh::Data layout (include/mesh/Data.hpp:13-35), vectorized with numpy.

Same node numbering, element-node order and boundary tags as BlockMesh2D/BlockMesh3D::generate
(src/mesh/generator/BlockMesh2D.cpp:37-117, src/mesh/generator/BlockMesh3D.cpp:26-139): nodes
x-fastest, element-local nodes x-fastest (tensor-product Lagrange order), faces tagged
LEFT/RIGHT/FRONT(BOTTOM in 2D)/BACK(TOP in 2D)/BOTTOM/TOP = 0..5, -1 for interior faces.
"""
import numpy as np


def block_mesh(nsd, nel, lo, hi, order):
    """Return (xyz, ien, rng) host arrays: xyz float64[nnodes*nsd], ien int64[nelem*npe], rng int32[nelem*nfaces]."""
    p = int(order)
    nx, ny = int(nel[0]), int(nel[1])
    nz = int(nel[2]) if nsd == 3 else 1
    NX, NY = nx * p + 1, ny * p + 1
    NZ = nz * p + 1 if nsd == 3 else 1
    dx = (hi[0] - lo[0]) / float(nx * p)
    dy = (hi[1] - lo[1]) / float(ny * p)
    i = np.arange(NX, dtype=np.float64)
    j = np.arange(NY, dtype=np.float64)
    if nsd == 2:
        X = np.broadcast_to(lo[0] + i * dx, (NY, NX))
        Y = np.broadcast_to((lo[1] + j * dy)[:, None], (NY, NX))
        xyz = np.stack([X.ravel(), Y.ravel()], axis=1).ravel()
    else:
        dz = (hi[2] - lo[2]) / float(nz * p)
        k = np.arange(NZ, dtype=np.float64)
        X = np.broadcast_to(lo[0] + i * dx, (NZ, NY, NX))
        Y = np.broadcast_to((lo[1] + j * dy)[None, :, None], (NZ, NY, NX))
        Z = np.broadcast_to((lo[2] + k * dz)[:, None, None], (NZ, NY, NX))
        xyz = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1).ravel()
    q = p + 1
    if nsd == 2:
        a = np.arange(q * q)
        ax, ay = a % q, a // q
        ey, ex = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        ex, ey = ex.ravel()[:, None], ey.ravel()[:, None]
        ien = (ey * p + ay[None, :]) * NX + (ex * p + ax[None, :])
        rng = np.full((nx * ny, 4), -1, np.int32)
        rng[:, 0] = np.where(ex[:, 0] == 0, 0, -1)
        rng[:, 1] = np.where(ex[:, 0] == nx - 1, 1, -1)
        rng[:, 2] = np.where(ey[:, 0] == 0, 2, -1)
        rng[:, 3] = np.where(ey[:, 0] == ny - 1, 3, -1)
    else:
        a = np.arange(q * q * q)
        ax, ay, az = a % q, (a // q) % q, a // (q * q)
        ez, ey, ex = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        ex, ey, ez = ex.ravel()[:, None], ey.ravel()[:, None], ez.ravel()[:, None]
        ien = (ez * p + az[None, :]) * (NY * NX) + (ey * p + ay[None, :]) * NX + (ex * p + ax[None, :])
        rng = np.full((nx * ny * nz, 6), -1, np.int32)
        rng[:, 0] = np.where(ex[:, 0] == 0, 0, -1)
        rng[:, 1] = np.where(ex[:, 0] == nx - 1, 1, -1)
        rng[:, 2] = np.where(ey[:, 0] == 0, 2, -1)
        rng[:, 3] = np.where(ey[:, 0] == ny - 1, 3, -1)
        rng[:, 4] = np.where(ez[:, 0] == 0, 4, -1)
        rng[:, 5] = np.where(ez[:, 0] == nz - 1, 5, -1)
    return np.ascontiguousarray(xyz), np.ascontiguousarray(ien.ravel().astype(np.int64)), np.ascontiguousarray(rng.ravel())
