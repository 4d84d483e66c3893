"""CPU tests of the oracle's overlap-mesh lid (interpolation.f90:10-69).

  - the vectorised restatement equals a node-by-node loop written in the
    order of the reference's statements, bit for bit;
  - the bilinear weights reproduce a field linear in x and y exactly (the
    field's value (i, j) taken at (i dx, j dy), as the reference's x1 = im dx
    places it), with the plane mean of u, v, p, indic and w's own plane;
  - the lid nodes cover the main mesh including its halo cells, never
    reading past them, for nr = 2 and 4.
"""
import math

import numpy as np
import pytest

import oracle as O

GRID = (16, 12, 10, 1 / 16, 1 / 12, 1 / 10)


def _fields(grid, seed):
    rng = np.random.default_rng(seed)
    shape = (grid[2] + 2, grid[1] + 2, grid[0] + 2)
    return [rng.normal(size=shape) for _ in range(5)]


def _loop(grid, nf, nr, fields):
    itot, jtot = grid[0], grid[1]
    lx, ly = itot * grid[3], jtot * grid[4]
    dx, dy = 1.0 / (itot / lx), 1.0 / (jtot / ly)
    dxc, dyc = 1.0 / ((itot * nr) / lx), 1.0 / ((jtot * nr) / ly)
    out = [np.zeros((jtot * nr + 2, itot * nr + 2)) for _ in range(5)]
    for i in range(itot * nr + 2):
        for j in range(jtot * nr + 2):
            xp = (i * dxc) + (.5 * (1. - (1. / nr)) * dx)
            yp = (j * dyc) + (.5 * (1. - (1. / nr)) * dy)
            x1 = math.floor(xp / dx) * dx
            x2 = (math.floor(xp / dx) + 1.) * dx
            y1 = math.floor(yp / dy) * dy
            y2 = (math.floor(yp / dy) + 1.) * dy
            c11 = ((x2 - xp) * (y2 - yp)) / ((x2 - x1) * (y2 - y1))
            c12 = ((x2 - xp) * (yp - y1)) / ((x2 - x1) * (y2 - y1))
            c21 = ((xp - x1) * (y2 - yp)) / ((x2 - x1) * (y2 - y1))
            c22 = ((xp - x1) * (yp - y1)) / ((x2 - x1) * (y2 - y1))
            im, jm = math.floor(xp / dx), math.floor(yp / dy)
            for q, f in enumerate(fields):
                if q == 2:
                    q11, q12, q21, q22 = f[nf + 1, jm, im], f[nf + 1, jm + 1, im], f[nf + 1, jm, im + 1], \
                        f[nf + 1, jm + 1, im + 1]
                else:
                    q11 = .5 * (f[nf, jm, im] + f[nf + 1, jm, im])
                    q12 = .5 * (f[nf, jm + 1, im] + f[nf + 1, jm + 1, im])
                    q21 = .5 * (f[nf, jm, im + 1] + f[nf + 1, jm, im + 1])
                    q22 = .5 * (f[nf, jm + 1, im + 1] + f[nf + 1, jm + 1, im + 1])
                out[q][j, i] = (c11 * q11) + (c12 * q12) + (c21 * q21) + (c22 * q22)
    return out


@pytest.mark.parametrize("nr", [2, 4])
def test_vectorised_equals_the_statement_loop(nr):
    f = _fields(GRID, 3)
    for a, b in zip(O.overlap_lid(GRID, 4, nr, *f), _loop(GRID, 4, nr, f)):
        assert np.array_equal(a, b)


def test_linear_fields_are_reproduced():
    itot, jtot, ktot, dx, dy, dz = GRID
    k, j, i = np.meshgrid(np.arange(ktot + 2), np.arange(jtot + 2), np.arange(itot + 2), indexing="ij")
    lin = 0.3 + 1.7 * (i * dx) - 0.9 * (j * dy) + 0.25 * k
    nf, nr = 5, 2
    out = O.overlap_lid(GRID, nf, nr, lin, lin, lin, lin, lin)
    ii = np.arange(itot * nr + 2)[None, :]
    jj = np.arange(jtot * nr + 2)[:, None]
    xp = ii * dx / nr + 0.5 * (1 - 1 / nr) * dx
    yp = jj * dy / nr + 0.5 * (1 - 1 / nr) * dy
    plane_mean = 0.3 + 1.7 * xp - 0.9 * yp + 0.25 * (nf + 0.5)
    face = 0.3 + 1.7 * xp - 0.9 * yp + 0.25 * (nf + 1)
    for q, o in enumerate(out):
        ref = face if q == 2 else plane_mean
        assert np.abs(o - ref).max() < 1e-13


@pytest.mark.parametrize("nr", [2, 4])
def test_nodes_stay_inside_the_halo(nr):
    itot, jtot = GRID[0], GRID[1]
    lx = itot * GRID[3]
    dx, dxc = 1.0 / (itot / lx), 1.0 / ((itot * nr) / lx)
    xp = np.arange(itot * nr + 2) * dxc + (0.5 * (1.0 - 1.0 / nr)) * dx
    im = np.floor(xp / dx)
    assert im.min() == 0 and im.max() + 1 <= itot + 1
