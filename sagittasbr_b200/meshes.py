"""Seeded synthetic PEC meshes for the benchmark and test workloads.

Every generator returns ``(verts float32 [V,3], tris uint32 [T,3])`` with the
winding pointing toward the illuminated side (outward for closed bodies, into the
octant for the trihedral's inner faces): the reference's PO term only counts hits
whose geometric normal ``unit(e1 x e2)`` faces the incoming ray
(src/cuda/poKernels.cu:92-94, src/cuda/rtKernels.cu:42), so winding changes
results.  Meshes are centred on their bounding-box centre because the reference
launcher square is centred on the world origin (src/app/sweep.cu:357-364).
"""
from __future__ import annotations

import math

import numpy as np

C0 = 299792458.0


def _orient_outward(verts, tris, centre=None):
    """Flip triangles whose normal points toward ``centre`` (closed convex-ish bodies)."""
    v = verts.astype(np.float64)
    c = v.mean(axis=0) if centre is None else np.asarray(centre, dtype=np.float64)
    a, b, cc = v[tris[:, 0]], v[tris[:, 1]], v[tris[:, 2]]
    n = np.cross(b - a, cc - a)
    cen = (a + b + cc) / 3.0 - c
    flip = np.einsum("ij,ij->i", n, cen) < 0
    out = tris.copy()
    out[flip, 1], out[flip, 2] = tris[flip, 2], tris[flip, 1]
    return out


def centre_on_aabb(verts):
    v = np.asarray(verts, dtype=np.float64)
    mid = 0.5 * (v.min(axis=0) + v.max(axis=0))
    return (v - mid).astype(np.float32)


def icosahedron():
    p = (1.0 + math.sqrt(5.0)) / 2.0
    raw = []
    for s1 in (-1.0, 1.0):
        for s2 in (-1.0, 1.0):
            raw += [(0.0, s1, s2 * p), (s1, s2 * p, 0.0), (s2 * p, 0.0, s1)]
    v = np.array(raw)
    # faces: vertex triples that are mutually one edge (length 2) apart
    d = np.linalg.norm(v[:, None] - v[None], axis=-1)
    adj = np.abs(d - 2.0) < 1e-9
    faces = []
    for i in range(12):
        for j in range(i + 1, 12):
            if not adj[i, j]:
                continue
            for k in range(j + 1, 12):
                if adj[i, k] and adj[j, k]:
                    faces.append((i, j, k))
    v = v / np.linalg.norm(v, axis=1, keepdims=True)
    t = _orient_outward(v, np.array(faces, dtype=np.int64), centre=(0, 0, 0))
    return v, t


def icosphere(level: int = 5, radius: float = 1.0):
    """Subdivided icosahedron: 20*4**level triangles on a sphere of ``radius``."""
    v, t = icosahedron()
    verts = [tuple(x) for x in v]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = np.add(verts[a], verts[b]) * 0.5
                m = m / np.linalg.norm(m)
                cache[key] = len(verts)
                verts.append(tuple(m))
            return cache[key]

        nt = []
        for a, b, c in t:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nt += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        t = np.array(nt, dtype=np.int64)
    V = np.array(verts) * radius
    return V.astype(np.float32), t.astype(np.uint32)


def _grid_plate(axis: int, offset: float, lo: float, hi: float, n: int):
    """Square plate in the plane x[axis] = offset spanning [lo,hi]^2, n x n x 2 triangles,
    normal along +axis.  Local coordinates a,b map to axes (axis+1)%3, (axis+2)%3."""
    s = np.linspace(lo, hi, n + 1)
    A, B = np.meshgrid(s, s, indexing="ij")  # A along a, B along b
    P = np.zeros(((n + 1) * (n + 1), 3))
    P[:, axis] = offset
    P[:, (axis + 1) % 3] = A.ravel()
    P[:, (axis + 2) % 3] = B.ravel()
    idx = np.arange((n + 1) * (n + 1)).reshape(n + 1, n + 1)
    p00 = idx[:-1, :-1].ravel()
    p10 = idx[1:, :-1].ravel()
    p11 = idx[1:, 1:].ravel()
    p01 = idx[:-1, 1:].ravel()
    t1 = np.stack([p00, p10, p11], axis=1)
    t2 = np.stack([p00, p11, p01], axis=1)
    T = np.empty((2 * n * n, 3), dtype=np.int64)
    T[0::2] = t1
    T[1::2] = t2
    return P, T


def trihedral(edge: float = 1.0, n: int = 100):
    """Three orthogonal square plates meeting at the corner (-edge/2,)*3, normals
    pointing into the +x,+y,+z octant; 3 * n*n*2 triangles."""
    h = edge / 2.0
    vs, ts, off = [], [], 0
    for axis in range(3):
        P, T = _grid_plate(axis, -h, -h, h, n)
        vs.append(P)
        ts.append(T + off)
        off += P.shape[0]
    return np.concatenate(vs).astype(np.float32), np.concatenate(ts).astype(np.uint32)


def plate(size: float = 1.0, n: int = 1, axis: int = 2):
    """Square plate in the plane through the origin normal to ``axis`` (facing +axis)."""
    P, T = _grid_plate(axis, 0.0, -size / 2, size / 2, n)
    return P.astype(np.float32), T.astype(np.uint32)


def dihedral(edge: float = 1.0, n: int = 4):
    """Two orthogonal plates (x = -edge/2 facing +x, y = -edge/2 facing +y)."""
    h = edge / 2.0
    vs, ts, off = [], [], 0
    for axis in (0, 1):
        P, T = _grid_plate(axis, -h, -h, h, n)
        vs.append(P)
        ts.append(T + off)
        off += P.shape[0]
    V = np.concatenate(vs)
    return centre_on_aabb(V), np.concatenate(ts).astype(np.uint32)


def box(size: float = 1.0):
    """Axis-aligned cube of side ``size`` centred on the origin, 12 outward triangles."""
    h = size / 2.0
    V = np.array([[x, y, z] for x in (-h, h) for y in (-h, h) for z in (-h, h)])
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    T = []
    for a, b, c, d in quads:
        T += [(a, b, c), (a, c, d)]
    T = _orient_outward(V, np.array(T, dtype=np.int64), centre=(0, 0, 0))
    return V.astype(np.float32), T.astype(np.uint32)


def _grid_tris(nu: int, nv: int, offset: int = 0, wrap_v: bool = False, flip: bool = False):
    """Two triangles per cell of an (nu+1) x (nv+1) vertex grid (row-major, u slow).
    With wrap_v the last column connects back to the first (nv columns of vertices)."""
    cols = nv if wrap_v else nv + 1
    u = np.arange(nu)[:, None]
    v = np.arange(nv)[None, :]
    a = offset + u * cols + v
    b = offset + (u + 1) * cols + v
    vn = (v + 1) % cols if wrap_v else v + 1
    c = offset + (u + 1) * cols + vn
    d = offset + u * cols + vn
    t1 = np.stack([a, b, c], axis=-1).reshape(-1, 3)
    t2 = np.stack([a, c, d], axis=-1).reshape(-1, 3)
    T = np.empty((t1.shape[0] * 2, 3), dtype=np.int64)
    T[0::2], T[1::2] = t1, t2
    if flip:
        T[:, [1, 2]] = T[:, [2, 1]]
    return T


def _orient_by_normal(V, T, want):
    """Flip the whole component if its mean normal disagrees with `want` (a vector
    field evaluated at the triangle centroids, pointing to the outside)."""
    a, b, c = V[T[:, 0]], V[T[:, 1]], V[T[:, 2]]
    n = np.cross(b - a, c - a)
    w = want((a + b + c) / 3.0)
    if np.einsum("ij,ij->", n, w) < 0:
        T = T[:, [0, 2, 1]]
    return T


def superellipsoid_fuselage(length: float = 20.0, radius: float = 1.5, n_eta: int = 1000, n_omega: int = 600,
                            e1: float = 0.3):
    """Closed body of revolution along x: x = L/2 s(eta)^e1, r = R c(eta)^e1 with
    s/c the signed powers of sin/cos (a superellipsoid blunted by e1 < 1); circular
    cross-section.  Poles are closed with triangle fans."""
    def spow(x, e):
        return np.sign(x) * np.abs(x) ** e
    eta = np.linspace(-np.pi / 2, np.pi / 2, n_eta + 1)[1:-1]   # interior rings
    om = np.linspace(0.0, 2 * np.pi, n_omega, endpoint=False)
    E, O = np.meshgrid(eta, om, indexing="ij")
    x = 0.5 * length * spow(np.sin(E), e1)
    r = radius * spow(np.cos(E), e1)
    V = np.stack([x, r * np.cos(O), r * np.sin(O)], axis=-1).reshape(-1, 3)
    nr = eta.size
    T = [_grid_tris(nr - 1, n_omega, 0, wrap_v=True)]
    tail = V.shape[0]
    nose = tail + 1
    V = np.concatenate([V, [[-0.5 * length, 0, 0], [0.5 * length, 0, 0]]])
    j = np.arange(n_omega)
    jn = (j + 1) % n_omega
    T.append(np.stack([np.full(n_omega, tail), jn, j], axis=1))
    last = (nr - 1) * n_omega
    T.append(np.stack([np.full(n_omega, nose), last + j, last + jn], axis=1))
    T = np.concatenate(T)
    T = _orient_by_normal(V, T, lambda p: p * np.array([0.0, 1.0, 1.0]))
    return V, T


def _naca_half_thickness(xi, t):
    """Half thickness of a symmetric 4-digit NACA section (closed trailing edge)."""
    return 5.0 * t * (0.2969 * np.sqrt(xi) - 0.1260 * xi - 0.3516 * xi ** 2 + 0.2843 * xi ** 3 - 0.1036 * xi ** 4)


def trapezoid_surface(span: float, root_chord: float, tip_chord: float, sweep_deg: float, thickness: float,
                      n_chord: int, n_span: int, origin, span_axis, thick_axis):
    """Closed swept trapezoidal lifting surface (upper + lower skins meeting at the
    leading and trailing edges, tip closed).  Chord along +x from the leading edge at
    `origin`; span along `span_axis` (unit vector); thickness along `thick_axis`."""
    xi = 0.5 * (1.0 - np.cos(np.linspace(0.0, np.pi, n_chord + 1)))    # cosine spacing
    eta = np.linspace(0.0, 1.0, n_span + 1)
    XI, ET = np.meshgrid(xi, eta, indexing="ij")
    chord = root_chord + (tip_chord - root_chord) * ET
    # the tip station is pinched to zero thickness so the two skins close there
    h = _naca_half_thickness(XI, thickness) * chord * np.minimum(1.0, (1.0 - ET) * n_span)
    xle = ET * span * np.tan(np.radians(sweep_deg))
    o = np.asarray(origin, dtype=np.float64)
    sa, ta = np.asarray(span_axis, float), np.asarray(thick_axis, float)
    base = o + (xle + XI * chord)[..., None] * np.array([1.0, 0, 0]) + (ET * span)[..., None] * sa
    up = (base + h[..., None] * ta).reshape(-1, 3)
    lo = (base - h[..., None] * ta).reshape(-1, 3)
    V = np.concatenate([up, lo])
    nv = up.shape[0]
    Tu = _grid_tris(n_chord, n_span, 0)
    Tl = _grid_tris(n_chord, n_span, nv, flip=True)
    # orient each skin so its normals point away from the chord plane
    Tu = _orient_by_normal(V, Tu, lambda p: np.broadcast_to(ta, p.shape))
    Tl = _orient_by_normal(V, Tl, lambda p: np.broadcast_to(-ta, p.shape))
    return V, np.concatenate([Tu, Tl])


def aircraft(seed: int = 1, jitter: float = 1e-3, fuselage=(1000, 600), wing=(100, 1000), tail=(50, 250)):
    """Seeded aircraft-like mesh (about 2.15 M triangles at the default resolution):
    superellipsoid fuselage 20 m long with 1.5 m semi-axes, swept trapezoidal wings
    (18 m span, chord 3 m -> 1 m, 25 deg sweep, 12 % thick), horizontal tail
    (6.4 m span) and a vertical fin, Gaussian vertex jitter (sigma = `jitter`),
    outward winding, centred on its bounding box."""
    parts = [superellipsoid_fuselage(20.0, 1.5, *fuselage)]
    nc, ns = wing
    for side in (1.0, -1.0):
        parts.append(trapezoid_surface(9.0, 3.0, 1.0, 25.0, 0.12, nc, ns, (-2.0, 0.0, -0.5), (0, side, 0), (0, 0, 1)))
    tc, ts = tail
    for side in (1.0, -1.0):
        parts.append(trapezoid_surface(3.2, 2.0, 0.8, 30.0, 0.10, tc, ts, (6.8, 0.0, 0.3), (0, side, 0), (0, 0, 1)))
    parts.append(trapezoid_surface(3.0, 2.5, 1.0, 35.0, 0.10, tc, ts, (6.5, 0.0, 0.9), (0, 0, 1), (0, 1, 0)))
    Vs, Ts, off = [], [], 0
    for V, T in parts:
        Vs.append(V)
        Ts.append(T + off)
        off += V.shape[0]
    V = np.concatenate(Vs)
    T = np.concatenate(Ts)
    if jitter > 0:
        V = V + np.random.default_rng(seed).normal(0.0, jitter, V.shape)
    return centre_on_aabb(V), T.astype(np.uint32)


def real_sph_harm(l: int, m: int, theta, phi):
    """Orthonormal real spherical harmonic Y_lm (theta polar from +z, phi azimuth)."""
    from scipy.special import lpmv
    am = abs(m)
    norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
    p = lpmv(am, l, np.cos(theta))
    if m == 0:
        return norm * p
    return math.sqrt(2.0) * norm * p * (np.cos(am * phi) if m > 0 else np.sin(am * phi))


def ellipsoid_sh(axes=(2.0, 1.0, 0.5), n_theta: int = 224, n_phi: int = 448, n_modes: int = 32,
                 sigma: float = 0.01, seed: int = 4):
    """Ellipsoid with the given semi-axes, tessellated on a (theta, phi) grid
    (2 n_phi (n_theta - 1) triangles: 199,808 at the defaults), each vertex moved
    radially by a seeded field sum_i a_i Y_i(theta, phi) over the first ``n_modes``
    real spherical harmonics (l = 0, 1, ...; m = -l..l), a_i ~ N(0, sigma) metres."""
    rng = np.random.default_rng(seed)
    modes = [(l, m) for l in range(16) for m in range(-l, l + 1)][:n_modes]
    amps = rng.normal(0.0, sigma, size=len(modes))
    th = np.linspace(0.0, np.pi, n_theta + 1)[1:-1]
    ph = np.linspace(0.0, 2 * np.pi, n_phi, endpoint=False)
    TH, PH = np.meshgrid(th, ph, indexing="ij")
    a, b, c = axes
    P = np.stack([a * np.sin(TH) * np.cos(PH), b * np.sin(TH) * np.sin(PH), c * np.cos(TH)], axis=-1)
    delta = sum(amp * real_sph_harm(l, m, TH, PH) for amp, (l, m) in zip(amps, modes))
    P = P + (delta / np.linalg.norm(P, axis=-1))[..., None] * P
    V = P.reshape(-1, 3)
    poles = []
    for pole_theta, z in ((0.0, c), (np.pi, -c)):
        d = sum(amp * real_sph_harm(l, m, np.array(pole_theta), np.array(0.0)) for amp, (l, m) in zip(amps, modes))
        poles.append([0.0, 0.0, z + np.sign(z) * float(d)])
    top, bottom = V.shape[0], V.shape[0] + 1
    V = np.concatenate([V, np.array(poles)])
    nr = th.size
    T = [_grid_tris(nr - 1, n_phi, 0, wrap_v=True)]
    j = np.arange(n_phi)
    jn = (j + 1) % n_phi
    T.append(np.stack([np.full(n_phi, top), j, jn], axis=1))
    last = (nr - 1) * n_phi
    T.append(np.stack([np.full(n_phi, bottom), last + jn, last + j], axis=1))
    T = np.concatenate(T)
    T = _orient_outward(V, T, centre=(0.0, 0.0, 0.0))
    return centre_on_aabb(V), T.astype(np.uint32)


def plate_cluster(n_plates: int, n: int, size: float = 0.5, spread: float = 1.0, seed: int = 0):
    """``n_plates`` square plates (side ``size``, n x n x 2 triangles each), randomly
    rotated and placed within a cube of side ``spread``; both faces are lit from
    the side their normal points to."""
    rng = np.random.default_rng(seed)
    vs, ts, off = [], [], 0
    for _ in range(n_plates):
        P, T = _grid_plate(2, 0.0, -size / 2, size / 2, n)
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        Rm = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                       [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                       [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        vs.append(P @ Rm.T + rng.uniform(-spread / 2, spread / 2, size=3))
        ts.append(T + off)
        off += P.shape[0]
    return centre_on_aabb(np.concatenate(vs)), np.concatenate(ts).astype(np.uint32)


def uneven_batch(n_meshes: int = 64, seed: int = 5, tri_range=(1_000, 500_000)):
    """Seeded batch of meshes of uneven cost: icospheres, trihedrals, jittered
    SH-displaced ellipsoids and plate clusters with log-uniform triangle counts in
    ``tri_range``; each instance has its own frequency (uniform 1-12 GHz), its own
    azimuth sweep (90-1440 angles at a random elevation), 2-6 bounces and its own
    aperture G = 2 R_bs with n = ceil(10 G f / c) rays per side.  Returns a list of
    dicts (verts, tris, kind, freq, theta, phi, max_bounces, G, n)."""
    rng = np.random.default_rng(seed)
    out = []
    lo, hi = np.log(tri_range[0]), np.log(tri_range[1])
    for i in range(n_meshes):
        kind = ("icosphere", "trihedral", "ellipsoid", "plates")[i % 4]
        target = float(np.exp(rng.uniform(lo, hi)))
        size = float(rng.uniform(0.3, 1.5))
        if kind == "icosphere":
            level = int(np.clip(round(np.log(target / 20.0) / np.log(4.0)), 2, 7))
            v, t = icosphere(level, size / 2)
        elif kind == "trihedral":
            v, t = trihedral(size, max(1, int(round(np.sqrt(target / 6.0)))))
        elif kind == "ellipsoid":
            nt = max(8, int(round(np.sqrt(target / 4.0))))
            v, t = ellipsoid_sh((size, 0.6 * size, 0.35 * size), n_theta=nt, n_phi=2 * nt, sigma=0.01 * size,
                                seed=int(rng.integers(1 << 30)))
            v = (v + rng.normal(0.0, 1e-3 * size, v.shape)).astype(np.float32)
        else:
            k = int(rng.integers(3, 9))
            n = max(1, int(round(np.sqrt(target / (2.0 * k)))))
            v, t = plate_cluster(k, n, size / 2, size, seed=int(rng.integers(1 << 30)))
        f = float(rng.uniform(1e9, 12e9))
        na = int(rng.integers(90, 1441))
        th0 = float(rng.uniform(30.0, 150.0))
        G = 2.0 * bounding_radius(v)
        out.append(dict(verts=v, tris=t, kind=kind, freq=f, theta=np.full(na, th0),
                        phi=np.linspace(0.0, 360.0, na, endpoint=False), max_bounces=int(rng.integers(2, 7)),
                        G=G, n=rays_for(f, G)))
    return out


def bounding_radius(verts) -> float:
    """Radius of the bounding sphere about the AABB centre."""
    v = np.asarray(verts, dtype=np.float64)
    mid = 0.5 * (v.min(axis=0) + v.max(axis=0))
    return float(np.sqrt(((v - mid) ** 2).sum(axis=1).max()))


def rays_for(freq_hz: float, grid_size: float, rays_per_wavelength: float = 10.0) -> int:
    """n_x = n_y = ceil(rays_per_wavelength * G / lambda)."""
    return int(math.ceil(rays_per_wavelength * grid_size * freq_hz / C0 - 1e-9))
