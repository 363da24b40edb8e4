"""Seeded synthetic scenes for the PPPM-TDBEM step: meshes, rigid motion, accelerations.

The benchmark configurations of this project are synthetic (no dataset is involved):
  static sphere   icosphere subdivision 3 (642 vertices, 1280 triangles), radius 0.1 m,
                  res 32, grid length 2x the bounding box, dt = 0.5 h / (sqrt(3) c),
                  uniform acceleration sin(2 pi 1000 t), listener at int(0.875 res)
  moving sphere   icosphere subdivision 4 (2562 / 5120) with seeded +-10% radial noise,
  + plate         radius 0.08 m, translating 0.05 sin(2 pi 3 t) m along x and rotating
                  2 rad/s about a seeded axis, plus a static 1280-triangle plate; res 64;
                  band-limited (100 Hz - 8 kHz) unit-RMS Gaussian per-vertex accelerations
                  averaged to triangles; motion frames sampled at 1 kHz
  batch           scenes drawn from one seed with res in {24, 32, 48, 64}, perturbed
                  icospheres of subdivision 2-4 and 1000-4000 steps
Grid placement follows the reference's demo driver (experiments/demo/main.cu:96-103): grid
centred on the scene bounding box, length = factor * longest box side, h = length / res,
and for moving scenes dt = 1 / int(1.01 / (h / sqrt(3) / c)).
"""
import math

import numpy as np

C_REF = 340.3  # AIR_WAVE_SPEED (macro.h:82)


def icosphere(subdivisions):
    """Unit icosphere: 10 * 4^n + 2 vertices, 20 * 4^n triangles (outward winding)."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, float) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts, np.float64), np.array(faces, np.int32)


def perturbed_sphere(subdivisions, radius, noise, rng):
    v, f = icosphere(subdivisions)
    r = radius * (1.0 + noise * rng.uniform(-1.0, 1.0, size=len(v)))
    return (v * r[:, None]).astype(np.float64), f


def plate(nx, nz, size_x, size_z, y):
    """Flat rectangle in the x-z plane at height y, nx * nz quads, 2 * nx * nz triangles."""
    xs = np.linspace(-size_x / 2, size_x / 2, nx + 1)
    zs = np.linspace(-size_z / 2, size_z / 2, nz + 1)
    X, Z = np.meshgrid(xs, zs, indexing="ij")
    verts = np.stack([X.ravel(), np.full(X.size, y), Z.ravel()], 1)
    f = []
    for i in range(nx):
        for k in range(nz):
            a, b = i * (nz + 1) + k, (i + 1) * (nz + 1) + k
            f += [(a, b + 1, b), (a, a + 1, b + 1)]
    return verts, np.array(f, np.int32)


def rotation_matrix(axis, angle):
    axis = np.asarray(axis, float) / np.linalg.norm(axis)
    x, y, z = axis
    c, s = math.cos(angle), math.sin(angle)
    C = 1 - c
    return np.array([[c + x * x * C, x * y * C - z * s, x * z * C + y * s],
                     [y * x * C + z * s, c + y * y * C, y * z * C - x * s],
                     [z * x * C - y * s, z * y * C + x * s, c + z * z * C]])


def grid_for_bbox(lo, hi, res, factor):
    """Grid of the demo driver: centred on the box, length = factor * longest side."""
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    length = float((hi - lo).max()) * factor
    h = length / res
    centre = (lo + hi) / 2
    min_pos = centre - length / 2
    return np.float32(h), min_pos.astype(np.float32)


def demo_dt(h, c=C_REF):
    """dt = 1 / int(1.01 / (h / sqrt(3) / c)) (experiments/demo/main.cu:103,128)."""
    frame_rate = int(np.float32(1.01) / (np.float32(h) / np.float32(math.sqrt(3)) / np.float32(c)))
    return np.float32(1.0 / frame_rate), frame_rate


def band_noise(n_series, n_steps, dt, lo_hz, hi_hz, rng):
    """Unit-RMS Gaussian noise band-limited to [lo_hz, hi_hz] by an FFT mask, per series."""
    x = rng.standard_normal((n_series, n_steps))
    X = np.fft.rfft(x, axis=1)
    freqs = np.fft.rfftfreq(n_steps, dt)
    X[:, (freqs < lo_hz) | (freqs > hi_hz)] = 0
    y = np.fft.irfft(X, n_steps, axis=1)
    rms = np.sqrt((y ** 2).mean(axis=1, keepdims=True))
    rms[rms == 0] = 1
    return (y / rms).astype(np.float32)


class StaticSphere:
    """Static pulsating sphere at res 32 (the reference's CPU-sized case)."""

    def __init__(self, res=32, subdivisions=3, radius=0.1, factor=2.0, steps=2000, freq=1000.0, c=C_REF):
        v, f = icosphere(subdivisions)
        self.verts = (v * radius).astype(np.float32)
        self.tris = f
        self.res = res
        self.h, self.min_pos = grid_for_bbox(self.verts.min(0), self.verts.max(0), res, factor)
        self.dt = np.float32(0.5 * self.h / (math.sqrt(3) * c))
        self.steps = steps
        self.freq = freq
        self.listener = (int(0.875 * res),) * 3

    def acc(self, first, count):
        t = (np.arange(first, first + count, dtype=np.float64)) * float(self.dt)
        a = np.sin(2 * math.pi * self.freq * t).astype(np.float32)
        return np.repeat(a[:, None], len(self.tris), 1)


class MovingScene:
    """Moving perturbed sphere plus a static plate (res 64, 1 kHz motion frames)."""

    def __init__(self, res=64, seed=7, subdivisions=4, radius=0.08, noise=0.1, amp=0.05, freq=3.0, omega=2.0,
                 plate_tris=1280, steps=8820, frame_hz=1000.0, factor=2.0, c=C_REF):
        rng = np.random.default_rng(seed)
        sv, sf = perturbed_sphere(subdivisions, radius, noise, rng)
        self.sphere_verts = sv
        self.axis = rng.standard_normal(3)
        self.axis /= np.linalg.norm(self.axis)
        nq = plate_tris // 2
        nx = 32 if nq % 32 == 0 else int(math.sqrt(nq))
        nz = nq // nx
        rmax = radius * (1 + noise)
        pv, pf = plate(nx, nz, 2 * (amp + rmax), 2 * rmax, -(rmax + 0.05))
        self.plate_verts = pv
        self.nsv = len(sv)
        self.tris = np.concatenate([sf, pf + len(sv)]).astype(np.int32)
        self.n_sphere_tris = len(sf)
        self.amp, self.freq, self.omega = amp, freq, omega
        lo = np.minimum(np.array([-amp - rmax, -rmax, -rmax]), pv.min(0))
        hi = np.maximum(np.array([amp + rmax, rmax, rmax]), pv.max(0))
        self.res = res
        self.h, self.min_pos = grid_for_bbox(lo, hi, res, factor)
        self.dt, self.frame_rate = demo_dt(self.h, c)
        self.steps = steps
        self.frame_hz = frame_hz
        self.listener = (int(0.875 * res),) * 3
        self.seed = seed
        self._noise = None

    def verts_at(self, time):
        R = rotation_matrix(self.axis, self.omega * time)
        sv = self.sphere_verts @ R.T
        sv[:, 0] += self.amp * math.sin(2 * math.pi * self.freq * time)
        return np.concatenate([sv, self.plate_verts]).astype(np.float32)

    def frame_of_step(self, step):
        """Motion frame in force at the start of PPPM step `step` (frame time <= t)."""
        return int(math.floor(step * float(self.dt) * self.frame_hz + 1e-9))

    def frame_verts(self, frame):
        return self.verts_at(frame / self.frame_hz)

    def acc(self, first, count):
        """Per-triangle accelerations for steps [first, first + count): sphere triangles carry
        band-limited vertex noise averaged to the triangle, the plate is silent."""
        need = first + count
        if self._noise is None or self._noise.shape[1] < need:
            n = max(need, self.steps)
            rng = np.random.default_rng(self.seed + 1)
            self._noise = band_noise(self.nsv, n, float(self.dt), 100.0, 8000.0, rng)
        vn = self._noise[:, first:need]
        sf = self.tris[: self.n_sphere_tris]
        tri = (vn[sf[:, 0]] + vn[sf[:, 1]] + vn[sf[:, 2]]) / np.float32(3)
        out = np.zeros((count, len(self.tris)), np.float32)
        out[:, : self.n_sphere_tris] = tri.T
        return out


def _bandpass_sos(lo_hz, hi_hz, fs, order=4):
    from scipy.signal import butter

    return butter(order, [lo_hz, hi_hz], btype="bandpass", fs=fs, output="sos")


class StreamedNoise:
    """Band-limited Gaussian noise for many series, generated in time order without holding the
    whole run: white noise in seeded blocks through a Butterworth band-pass whose state carries
    over between blocks, scaled to unit RMS by the filter's noise gain.  Any step range can be
    asked for; a range before the last one restarts from step 0 (same values)."""

    BLOCK = 512

    def __init__(self, n_series, dt, lo_hz, hi_hz, seed):
        from scipy.signal import sosfilt, sosfilt_zi  # noqa: F401

        self.n, self.seed = n_series, seed
        self.sos = _bandpass_sos(lo_hz, hi_hz, 1.0 / float(dt))
        imp = np.zeros(1 << 17)
        imp[0] = 1.0
        from scipy.signal import sosfilt

        self.gain = float(np.sqrt((sosfilt(self.sos, imp) ** 2).sum()))
        self._reset()

    def _reset(self):
        self.zi = np.zeros((self.sos.shape[0], self.n, 2))
        self.pos = 0
        self.buf = np.zeros((self.n, 0), np.float32)
        self.buf0 = 0

    def _block(self, b):
        from scipy.signal import sosfilt

        x = np.random.default_rng([self.seed, b]).standard_normal((self.n, self.BLOCK))
        y, self.zi = sosfilt(self.sos, x, axis=1, zi=self.zi)
        return (y / self.gain).astype(np.float32)

    def get(self, first, count):
        """(n_series, count) noise for steps [first, first + count)."""
        if first < self.buf0:
            self._reset()
        while self.pos < first + count:
            blk = self._block(self.pos // self.BLOCK)
            keep0 = min(max(self.buf0, first), self.pos)  # drop what lies before the request
            self.buf = np.concatenate([self.buf[:, keep0 - self.buf0:], blk], 1)
            self.buf0 = keep0
            self.pos += self.BLOCK
        return self.buf[:, first - self.buf0: first - self.buf0 + count]


class LargeScene:
    """Two moving perturbed icospheres (subdivision 5, 20480 triangles each) at res 128.

    Each sphere (radius 0.1 m, seeded +-10% radial noise) sits at x = -+0.17 m and follows its
    own seeded rigid trajectory: translation a sin(2 pi f t + phase) along a random direction
    (a in [0.02, 0.04] m, f in [1, 4] Hz) and rotation at omega in [1, 3] rad/s about a random
    axis.  The spheres stay more than 4 cells apart, so no face pair joins them.  The grid is
    centred on the box the motion can reach, length 1.5 x its longest side (h ~ 7.5 mm), which
    keeps every 3^3 list below 256 and every 4^3 list below 512 triangles (the reference's
    fixed capacities, particle_grid.h:9-11).  Both spheres carry per-vertex band-limited
    (100 Hz - 8 kHz) unit-RMS Gaussian accelerations averaged to triangles; motion frames at
    1 kHz; dt as in the demo driver; 20000 steps."""

    def __init__(self, res=128, seed=23, subdivisions=5, radius=0.1, noise=0.1, sep=0.17, factor=1.5, steps=20000,
                 frame_hz=1000.0, c=C_REF):
        rng = np.random.default_rng(seed)
        self.bodies = []
        verts, tris = [], []
        nv = 0
        for k, cx in enumerate((-sep, sep)):
            v, f = perturbed_sphere(subdivisions, radius, noise, rng)
            d = rng.standard_normal(3)
            ax = rng.standard_normal(3)
            body = dict(verts=v, centre=np.array([cx, 0.0, 0.0]), dir=d / np.linalg.norm(d),
                        axis=ax / np.linalg.norm(ax), amp=float(rng.uniform(0.02, 0.04)),
                        freq=float(rng.uniform(1.0, 4.0)), phase=float(rng.uniform(0, 2 * math.pi)),
                        omega=float(rng.uniform(1.0, 3.0)))
            self.bodies.append(body)
            verts.append(v)
            tris.append(f + nv)
            nv += len(v)
        self.tris = np.concatenate(tris).astype(np.int32)
        self.nv = nv
        rmax = radius * (1 + noise)
        lo = np.min([b["centre"] - b["amp"] - rmax for b in self.bodies], 0)
        hi = np.max([b["centre"] + b["amp"] + rmax for b in self.bodies], 0)
        self.res = res
        self.h, self.min_pos = grid_for_bbox(lo, hi, res, factor)
        self.dt, self.frame_rate = demo_dt(self.h, c)
        self.steps = steps
        self.frame_hz = frame_hz
        self.listener = (int(0.875 * res),) * 3
        self.seed = seed
        self._noise = StreamedNoise(nv, float(self.dt), 100.0, 8000.0, seed + 1)

    def verts_at(self, time):
        out = []
        for b in self.bodies:
            R = rotation_matrix(b["axis"], b["omega"] * time)
            v = b["verts"] @ R.T
            v += b["centre"] + b["dir"] * (b["amp"] * math.sin(2 * math.pi * b["freq"] * time + b["phase"]))
            out.append(v)
        return np.concatenate(out).astype(np.float32)

    def frame_of_step(self, step):
        return int(math.floor(step * float(self.dt) * self.frame_hz + 1e-9))

    def frame_verts(self, frame):
        return self.verts_at(frame / self.frame_hz)

    def acc(self, first, count):
        vn = self._noise.get(first, count)
        f = self.tris
        return ((vn[f[:, 0]] + vn[f[:, 1]] + vn[f[:, 2]]) / np.float32(3)).T.copy()


def frame_ranges(scene, nframes):
    """Step range [a, b) of each of the first nframes + 1 motion frames of a moving scene."""
    need = int(math.ceil((nframes + 1) / scene.frame_hz / float(scene.dt))) + 2
    start = [None] * (nframes + 2)
    for s in range(need):
        fr = scene.frame_of_step(s)
        if fr <= nframes + 1 and start[fr] is None:
            start[fr] = s
    return [(start[fr], start[fr + 1]) for fr in range(nframes + 1)]


def batch_scenes(n=64, seed=11, c=C_REF):
    """Independent scenes drawn from one seed: (res, verts, tris, h, min_pos, dt, steps)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        res = int(rng.choice([24, 32, 48, 64]))
        sub = int(rng.integers(2, 5))
        v, f = perturbed_sphere(sub, 0.1, 0.1, rng)
        v = v.astype(np.float32)
        h, mn = grid_for_bbox(v.min(0), v.max(0), res, 2.0)
        dt = np.float32(0.5 * h / (math.sqrt(3) * c))
        steps = int(rng.integers(1000, 4001))
        out.append(dict(res=res, verts=v, tris=f, h=h, min_pos=mn, dt=dt, steps=steps, freq=float(rng.uniform(500, 2000))))
    return out


def scene_cost(spec):
    """Estimated device work of one batch scene for sharding: steps x (grid cells + face-pair
    bytes in cell units).  The face pairs of a closed surface of T triangles spanning about half
    the grid: each centre sees the triangles of the ~16 surface cells of its 4^3 block, and the
    surface covers ~4 pi (res / 4)^2 cells, so P4 ~ 16 T^2 / (pi res^2 / 4); a face pair moves
    76 bytes against 12 per grid cell."""
    res, nt = spec["res"], len(spec["tris"])
    p4 = 16.0 * nt * nt / (math.pi * res * res / 4.0)
    return float(spec["steps"]) * (res ** 3 + p4 * 76.0 / 12.0)


def shard_by_cost(specs, world):
    """Static partition of batch scenes over `world` ranks: longest-processing-time-first by
    scene_cost (ties by index).  Returns one ascending index list per rank."""
    order = sorted(range(len(specs)), key=lambda i: (-scene_cost(specs[i]), i))
    load = [0.0] * world
    shards = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += scene_cost(specs[i])
    return [sorted(s) for s in shards]
