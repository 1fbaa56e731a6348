"""TEST INFRASTRUCTURE ONLY: a numpy restatement of the library's
single-precision filter (omega_h_v1_b200/csrc/common.cuh: tet_quality_f32,
edge_ratio_side_f32) beside the double values the reference computes, so the
filter's error bound can be checked on the CPU over many inputs.

* the estimates are evaluated in numpy float32 with the device code's
  operation order; with no fused multiply-add on the device (-fmad=false)
  and IEEE float division and square root on both sides, they are the
  device's values bit for bit (the GPU tests compare);
* the bound is the same formula evaluated in float64 (round to nearest) from
  those float32 intermediates: within about 2^-50 relative of the exact
  real value, which the device evaluates rounding every step upward;
* tet_quality64 is the reference's tet_quality (quality.hpp:68-89,
  size.hpp:14-46) in its operation order, in float64, and
  edge_ratio64 its metric edge length (size.cpp:57-69).

Nothing in the product imports this module.
"""
import numpy as np

F32 = np.float32
U = 2.0 ** -24


def perfect_tet_quality():
    """quality.hpp:15-18, formed as the reference forms it."""
    s = np.sqrt(np.sqrt(3.0) / 4.0)
    return (np.sqrt(2.0) / 12.0) / (s * s * s)


def _dot3(a, b):
    d = a[..., 0] * b[..., 0]
    d = d + a[..., 1] * b[..., 1]
    return d + a[..., 2] * b[..., 2]


def _dot3_ref(a, b):
    """dot3 (algebra.hpp): a running sum from 0."""
    d = 0.0 + a[..., 0] * b[..., 0]
    d = d + a[..., 1] * b[..., 1]
    return d + a[..., 2] * b[..., 2]


def _cross3(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def _tri_area64(x0, x1, x2):
    c = _cross3(x1 - x0, x2 - x0)
    return np.sqrt(_dot3_ref(c, c)) / 2.0


def tet_quality64(x):
    """x: (n, 4, 3) float64 -> the reference's tet_quality, bit for bit."""
    x = np.asarray(x, np.float64)
    x0, x1, x2, x3 = x[:, 0], x[:, 1], x[:, 2], x[:, 3]
    s = np.zeros(x.shape[0])
    for a in (_tri_area64(x0, x1, x2), _tri_area64(x1, x0, x3),
              _tri_area64(x2, x1, x3), _tri_area64(x0, x2, x3)):
        s = s + a * a
    arms = np.sqrt(s / 4.0)
    v = _dot3_ref(_cross3(x1 - x0, x2 - x0), x3 - x0) / 6.0
    r = np.sqrt(arms)
    q = v / (r * r * r)
    return q / perfect_tet_quality()


def tet_quality32(x):
    """(estimate float32, bound float64 with inf where the device gives none,
    intermediates) for x: (n, 4, 3) float64, in the device's order."""
    x = np.asarray(x, np.float64)
    with np.errstate(all="ignore"):
        d0 = (x[:, 1] - x[:, 0]).astype(F32)
        d1 = (x[:, 2] - x[:, 0]).astype(F32)
        d2 = (x[:, 3] - x[:, 0]).astype(F32)
        e12, e13, e23 = d1 - d0, d2 - d0, d2 - d1
        c0, c1, c2, c3 = _cross3(d0, d1), _cross3(d0, e13), _cross3(e12, e23), _cross3(d1, d2)
        s = _dot3(c0, c0) + _dot3(c1, c1)
        s = s + _dot3(c2, c2)
        s = s + _dot3(c3, c3)
        arms = np.sqrt(s * F32(0.0625))
        r = np.sqrt(arms)
        k6 = F32(6.0 * perfect_tet_quality())
        den = r * r * r * k6
        v6 = _dot3(c0, d2)
        q = v6 / den
        n0, n1, n2 = _dot3(d0, d0), _dot3(d1, d1), _dot3(d2, d2)
        lmax2 = np.maximum(np.maximum(np.maximum(n0, n1), np.maximum(n2, _dot3(e12, e12))),
                           np.maximum(_dot3(e13, e13), _dot3(e23, e23)))
        # the bound, in float64 from the float32 values
        S, L2, D = s.astype(np.float64), lmax2.astype(np.float64), den.astype(np.float64)
        eps = 9.0 * U * L2
        t = 7.0 * U * S + 4.0 * eps * np.sqrt(S) + 4.0 * eps * eps
        delta = t / S
        rho = (delta + 9.0 * U) * (1.0 + 10.0 * U)
        rho = rho * (1.0 + 2.0 * U) + U
        nn = n0.astype(np.float64) * n1.astype(np.float64) * n2.astype(np.float64)
        e = 13.0 * U * np.sqrt(nn) / D
        b = (rho * np.abs(q.astype(np.float64)) + e) / (1.0 - rho)
        b = b * (1.0 + 2.0 ** -20) + 2.0 ** -60
        ok = ((L2 >= 2.0 ** -40) & (L2 <= 2.0 ** 40) & (D > 0) & (S > 0) &
              np.isfinite(q) & (delta <= 0.125) & (rho <= 0.25) & (b <= 1.0))
        bound = np.where(ok, b, np.inf)
    return q, bound


def edge_ratio64(xa, xb, ha, hb):
    """size.cpp:57-69 in float64: sqrt(sum d^2) / ((ha + hb) / 2)."""
    d = xb - xa
    s = np.zeros(d.shape[0])
    for k in range(3):
        s = s + d[:, k] * d[:, k]
    return np.sqrt(s) / ((ha + hb) / 2)


def edge_ratio_side32(xa, xb, ha, hb, thr):
    """The device's +1 / -1 / 0 decision (edge_ratio_side_f32)."""
    with np.errstate(all="ignore"):
        d = (xb - xa).astype(F32)
        s = _dot3(d, d)
        hv = ((ha + hb) / 2).astype(F32)
        ok = (s >= F32(2.0 ** -100)) & (s <= F32(2.0 ** 100)) & \
             (hv >= F32(2.0 ** -100)) & (hv <= F32(2.0 ** 100))
        r = (np.sqrt(s) / hv).astype(np.float64)
        side = np.where(r * (1.0 - 6.0 * U) > thr, 1, np.where(r * (1.0 + 6.0 * U) < thr, -1, 0))
    return np.where(ok, side, 0).astype(np.int32)


# -- seeded stress inputs ------------------------------------------------------

def _regular(n, rng):
    base = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], np.float64)
    # random rotations from normalised Gaussian quaternions
    qv = rng.normal(size=(n, 4))
    qv /= np.linalg.norm(qv, axis=1, keepdims=True)
    w, a, b, c = qv.T
    R = np.stack([np.stack([1 - 2 * (b * b + c * c), 2 * (a * b - c * w), 2 * (a * c + b * w)], -1),
                  np.stack([2 * (a * b + c * w), 1 - 2 * (a * a + c * c), 2 * (b * c - a * w)], -1),
                  np.stack([2 * (a * c - b * w), 2 * (b * c + a * w), 1 - 2 * (a * a + b * b)], -1)],
                 axis=1)
    return np.einsum("nij,kj->nki", R, base)


def stress_tets(n, seed):
    """n seeded tets mixing the shapes that stress the bound: uniform random
    points, rotated regular tets at scales 1e-6..1e6 and far from the origin,
    slivers (four nearly coplanar points), needles and caps (a vertex close
    to another or to a face), shapes whose quality is near the 0.3 floor,
    edge-length ratios up to 1e4, and inverted copies."""
    rng = np.random.default_rng(seed)
    kinds = rng.integers(0, 8, size=n)
    out = np.empty((n, 4, 3))
    for k in range(8):
        idx = np.nonzero(kinds == k)[0]
        m = idx.size
        if m == 0:
            continue
        if k == 0:
            x = rng.random((m, 4, 3))
        elif k == 1:
            scale = 10.0 ** rng.uniform(-6, 6, size=(m, 1, 1))
            shift = (10.0 ** rng.uniform(-1, 4, size=(m, 1, 1))) * rng.normal(size=(m, 1, 3))
            x = _regular(m, rng) * scale + shift
        elif k == 2:  # slivers: a square with two opposite corners lifted by h
            h = 10.0 ** rng.uniform(-8, 0, size=m)
            sq = np.array([[0, 0, 0], [1, 1, 0], [1, 0, 0], [0, 1, 0]], np.float64)
            x = np.repeat(sq[None], m, 0)
            x[:, 0, 2] = h
            x[:, 1, 2] = h
            x = x + 1e-3 * rng.normal(size=(m, 4, 3)) * h[:, None, None]
        elif k == 3:  # needles: vertex 1 close to vertex 0
            x = _regular(m, rng)
            t = 10.0 ** rng.uniform(-8, 0, size=(m, 1))
            x[:, 1] = x[:, 0] + t * (x[:, 1] - x[:, 0])
        elif k == 4:  # caps: vertex 3 close to the face of the others
            x = _regular(m, rng)
            cen = x[:, :3].mean(axis=1)
            t = 10.0 ** rng.uniform(-8, 0, size=(m, 1))
            x[:, 3] = cen + t * (x[:, 3] - cen)
        elif k == 5:  # quality near 0.3: a regular tet flattened towards a plane
            x = _regular(m, rng)
            t = rng.uniform(0.15, 0.45, size=(m, 1))
            x[:, :, 2] *= t
        elif k == 6:  # edge-length ratios up to 1e4: anisotropic stretch
            x = rng.random((m, 4, 3))
            x[:, :, 0] *= 10.0 ** rng.uniform(0, 4, size=(m, 1))
        else:  # perturbed box cells, as meshes hold them
            x = _regular(m, rng) * 0.05 + 0.01 * rng.normal(size=(m, 4, 3)) + rng.random((m, 1, 3))
        out[idx] = x
    inv = rng.random(n) < 0.1
    out[inv] = out[inv][:, [1, 0, 2, 3]]
    return out


def stress_edges(n, seed, thr):
    """n seeded edges (end points, sizes) whose metric length is spread
    around thr, a quarter of them within a few float ulps of it."""
    rng = np.random.default_rng(seed)
    xa = rng.random((n, 3)) * 10.0 ** rng.uniform(-3, 3, size=(n, 1))
    dirn = rng.normal(size=(n, 3))
    dirn /= np.linalg.norm(dirn, axis=1, keepdims=True)
    length = 10.0 ** rng.uniform(-4, 1, size=n)
    xb = xa + dirn * length[:, None]
    ratio = np.where(rng.random(n) < 0.25,
                     thr * (1.0 + rng.integers(-24, 25, size=n) * U),
                     thr * 10.0 ** rng.uniform(-0.3, 0.3, size=n))
    w = length / ratio
    split = rng.uniform(0.2, 0.8, size=n)
    ha, hb = 2 * w * split, 2 * w * (1 - split)
    return xa, xb, ha, hb
