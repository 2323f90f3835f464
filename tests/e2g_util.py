"""Extend-to-grid target sets and masks, built from a grid's band data exactly
as the reference drivers select them (test helpers, used with the oracle)."""
import math

import numpy as np

CTR = 1.5  # E2G/utilities.h:19
AXES = (1.0, 0.5, 0.5)  # E2G/utilities.h:12-14


def stokeslet_density(pt):
    """stokeslet_density: E2G/utilities.cpp:267-285 (same operation order)."""
    x = pt[0] - CTR
    a, b = AXES[0], AXES[1]
    a_sq, b_sq = a * a, b * b
    x_sq = x * x
    e_sq = 1.0 - b_sq / a_sq
    e = math.sqrt(e_sq)
    Le = math.log((1.0 + e) / (1.0 - e))
    f0 = 4.0 * e_sq * e * a / b / ((1.0 + e_sq) * Le - 2.0 * e) / math.sqrt(a_sq - e_sq * x_sq)
    return (f0, 0.0, 0.0)


def phi(x, y, z):
    """phi (ellipsoid): E2G/utilities.cpp:10-29."""
    u, v, w = x - CTR, y - CTR, z - CTR
    return u * u / (AXES[0] ** 2) + v * v / (AXES[1] ** 2) + w * w / (AXES[2] ** 2) - 1.0


def face_targets(N, h):
    """Box-face points in the loop order of E2G/main.cpp:1058-1075."""
    pts, idx = [], []
    for i in range(N + 1):
        for j in range(N + 1):
            for k in range(N + 1):
                if i == 0 or i == N or j == 0 or j == N or k == 0 or k == N:
                    pts += [i * h, j * h, k * h]
                    idx.append((i * (N + 1) + j) * (N + 1) + k)
    return np.array(pts), np.array(idx)


def band_targets(N, h, nrst, b, x0, n0):
    """Band points evaluated with the regularized sums (E2G/main.cpp:1133-1162):
    interior, tagged, outside or on the surface. Returns xyz, b, x0, n0, f0, grid index."""
    xs, bs, x0s, n0s, f0s, gi = [], [], [], [], [], []
    M = N + 1
    for i in range(1, N):
        for j in range(1, N):
            for k in range(1, N):
                g = (i * M + j) * M + k
                ind = nrst[g]
                if ind == -1:
                    continue
                bb = b[ind]
                if bb > 0.0 or abs(bb) < 1e-12:
                    xs += [i * h, j * h, k * h]
                    bs.append(bb)
                    p0 = x0[3 * ind:3 * ind + 3]
                    x0s += list(p0)
                    n0s += list(n0[3 * ind:3 * ind + 3])
                    f0s += list(stokeslet_density(p0))
                    gi.append(g)
    return (np.array(xs), np.array(bs), np.array(x0s), np.array(n0s), np.array(f0s), np.array(gi))


def masks(N, h, nrst, band2):
    """BAND2 mask and the exterior-outside-BAND2 mask (E2G/main.cpp:1611-1614, 1654-1672)."""
    M = N + 1
    b2 = np.zeros(M ** 3, np.uint8)
    out = np.zeros(M ** 3, np.uint8)
    for i in range(M):
        for j in range(M):
            for k in range(M):
                g = (i * M + j) * M + k
                ind = nrst[g]
                if ind != -1 and band2[ind]:
                    b2[g] = 1
                if phi(i * h, j * h, k * h) > 0:
                    if ind == -1 or not band2[ind]:
                        out[g] = 1
    return b2, out
