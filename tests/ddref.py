"""Test helpers for the domain-decomposed dslash: qcu's rank grid restated
(include/lattice_set.h:89-95: t fastest, rank = ((gx*Gy+gy)*Gz+gz)*Gt+gt),
and the scatter / gather of PyQuda-layout fields between a global lattice
and the ranks' sub-lattices."""
import numpy as np


def coord_of(rank, grid):
    gx, gy, gz, gt = grid
    return [rank // gt // gz // gy, rank // gt // gz % gy, rank // gt % gz, rank % gt]


def eo_to_lex(f, latt):
    """[2, Lt, Lz, Ly, Lx/2, ...] (even-odd) -> [Lt, Lz, Ly, Lx, ...]."""
    Lx, Ly, Lz, Lt = latt
    out = np.empty((Lt, Lz, Ly, Lx) + f.shape[5:], f.dtype)
    t, z, y, x = np.meshgrid(np.arange(Lt), np.arange(Lz), np.arange(Ly), np.arange(Lx), indexing="ij")
    p = (x + y + z + t) & 1
    out[t, z, y, x] = f[p, t, z, y, x >> 1]
    return out


def lex_to_eo(g, latt):
    Lx, Ly, Lz, Lt = latt
    out = np.empty((2, Lt, Lz, Ly, Lx // 2) + g.shape[4:], g.dtype)
    t, z, y, x = np.meshgrid(np.arange(Lt), np.arange(Lz), np.arange(Ly), np.arange(Lx), indexing="ij")
    out[(x + y + z + t) & 1, t, z, y, x >> 1] = g[t, z, y, x]
    return out


def block(lex, c, loc):
    """The sub-lattice at grid coordinate c (local extents loc) of a lex field."""
    Lx, Ly, Lz, Lt = loc
    return lex[c[3] * Lt:(c[3] + 1) * Lt, c[2] * Lz:(c[2] + 1) * Lz, c[1] * Ly:(c[1] + 1) * Ly,
               c[0] * Lx:(c[0] + 1) * Lx]


def scatter_spinor(full_eo, glatt, loc, grid):
    """Global full spinor -> [ranks, 2, ...local half shape...]."""
    lex = eo_to_lex(full_eo, glatt)
    n = int(np.prod(grid))
    return np.stack([lex_to_eo(block(lex, coord_of(r, grid), loc), loc) for r in range(n)])


def scatter_gauge(U, glatt, loc, grid):
    """Global gauge [4, 2, ...] -> [ranks, 4, 2, ...local...]."""
    lex = [eo_to_lex(U[d], glatt) for d in range(4)]
    n = int(np.prod(grid))
    return np.stack([np.stack([lex_to_eo(block(lex[d], coord_of(r, grid), loc), loc) for d in range(4)])
                     for r in range(n)])


def gather_half(local_halves, parity, glatt, loc, grid):
    """Ranks' half spinors of one parity -> the global half spinor of that parity."""
    Lx, Ly, Lz, Lt = glatt
    lex = np.zeros((Lt, Lz, Ly, Lx) + local_halves.shape[-2:], local_halves.dtype)
    for r in range(local_halves.shape[0]):
        c = coord_of(r, grid)
        full = np.zeros((2,) + local_halves.shape[1:], local_halves.dtype)
        full[parity] = local_halves[r]
        sub = eo_to_lex(full, loc)
        blk = block(lex, c, loc)
        t, z, y, x = np.meshgrid(*[np.arange(n) for n in (loc[3], loc[2], loc[1], loc[0])], indexing="ij")
        mask = ((x + y + z + t) & 1) == parity  # local parity = global parity (even extents)
        blk[mask] = sub[mask]
    return lex_to_eo(lex, glatt)[parity]
