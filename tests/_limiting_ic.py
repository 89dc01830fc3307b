"""Initial states with discontinuities for the limiting ADER-DG tests: nodal
values on the Gauss-Legendre nodes of a 2D grid (cells x fastest,
per cell [y][x][variable]), 5 Euler variables, gamma = 1.4."""
import numpy as np

GAMMA = 1.4


def nodes(order):
    return (np.polynomial.legendre.leggauss(order + 1)[0] + 1) / 2


def explosion(order, n, length=(1.0, 1.0), radius=0.25, inner=(1.0, 1.0), outer=(0.125, 0.1), center=(0.5, 0.5)):
    """Cylindrical explosion: (density, pressure) = inner inside the circle,
    outer outside, at rest."""
    xi = nodes(order)
    B = order + 1
    nx, ny = n
    hx, hy = length[0] / nx, length[1] / ny
    X = (np.arange(nx)[None, :, None, None] + xi[None, None, None, :]) * hx
    Y = (np.arange(ny)[:, None, None, None] + xi[None, None, :, None]) * hy
    X, Y = np.broadcast_arrays(X, Y)  # [cy][cx][iy][ix]
    r2 = (X - center[0]) ** 2 + (Y - center[1]) ** 2
    inside = r2 < radius ** 2
    rho = np.where(inside, inner[0], outer[0])
    p = np.where(inside, inner[1], outer[1])
    q = np.zeros(X.shape + (5,))
    q[..., 0] = rho
    q[..., 4] = p / (GAMMA - 1)
    # [cy][cx][iy][ix][v] is cells x fastest, nodes [y][x] per cell
    return q.reshape(ny * nx * B * B * 5)


def smooth(order, n, length=(1.0, 1.0), amp=0.1):
    """Density wave advected diagonally: a state the DMP leaves alone."""
    xi = nodes(order)
    nx, ny = n
    hx, hy = length[0] / nx, length[1] / ny
    X = (np.arange(nx)[None, :, None, None] + xi[None, None, None, :]) * hx
    Y = (np.arange(ny)[:, None, None, None] + xi[None, None, :, None]) * hy
    X, Y = np.broadcast_arrays(X, Y)
    rho = 1.0 + amp * np.sin(2 * np.pi * (X + Y))
    q = np.zeros(X.shape + (5,))
    q[..., 0] = rho
    q[..., 1] = rho
    q[..., 2] = rho
    q[..., 4] = 1.0 / (GAMMA - 1) + 0.5 * 2 * rho
    return q.reshape(-1)


def explosion3d(order, n, radius=0.25, inner=(1.0, 1.0), outer=(0.125, 0.1), center=(0.5, 0.5, 0.5)):
    """Spherical explosion in the unit cube (cells x fastest, per cell
    [z][y][x][variable])."""
    xi = nodes(order)
    nx, ny, nz = n
    B = order + 1
    X = (np.arange(nx)[None, None, :, None, None, None] + xi[None, None, None, None, None, :]) / nx
    Y = (np.arange(ny)[None, :, None, None, None, None] + xi[None, None, None, None, :, None]) / ny
    Z = (np.arange(nz)[:, None, None, None, None, None] + xi[None, None, None, :, None, None]) / nz
    X, Y, Z = np.broadcast_arrays(X, Y, Z)  # [cz][cy][cx][iz][iy][ix]
    inside = (X - center[0]) ** 2 + (Y - center[1]) ** 2 + (Z - center[2]) ** 2 < radius ** 2
    q = np.zeros(X.shape + (5,))
    q[..., 0] = np.where(inside, inner[0], outer[0])
    q[..., 4] = np.where(inside, inner[1], outer[1]) / (GAMMA - 1)
    return q.reshape(nz * ny * nx * B ** 3 * 5)
