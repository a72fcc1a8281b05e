"""Seeded analytic irradiance fields: the stand-in for BallaSim's renderer on this path.

The renderer (src/render, ray tracing) is outside this package. In its place the sampler evaluates one of two
closed-form fields of irradiance E(x, y, t) (renderer units, photocurrent = illuminance_scale x E fA) on the
device, at the pixel centre (x + 0.5, y + 0.5), with every signature 0:

- ``tanh_edge``: E = base + amp tanh((n . p - speed t - c) / width), a straight edge moving along its normal n.
- ``blobs``: E = base + sum_k A_k exp(-|p - c_k(t)|^2 / (2 r_k^2)) with c_k(t) = c_k(0) + v_k t; a blob adds
  exactly 0 beyond 6 r_k (its term is below fp32 resolution there), which lets the device cull it per tile.

Both are evaluated in fp32 in a fixed operation order with the project's own deterministic exp, so that the
device and any CPU evaluation agree bit for bit. The parameters are drawn here from a SplitMix64 stream of the
seed (Vigna's published mixer): uniforms (z >> 11) 2^-53, normals by Box-Muller.

Level rule (the planner's ``clamp(ceil(log2(v W / d_px)), l_min, l_max)``, src/engine/motion.cpp:1330-1338, with
d_px = 0.25 px, src/engine/engine.h:61): v is the speed of the fastest blob whose 3 r support covers the pixel at
the window start (none: l_min); the tanh edge takes l_min.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

BLOB_WORDS = 10  # a, cx0, cy0, vx, vy, 1/(2 r^2), (6 r)^2, (3 r)^2, |v|, pad
KIND_TANH_EDGE = 1
KIND_BLOBS = 2


class SplitMix64:
    """SplitMix64 (Steele, Lea, Flood 2014; Vigna's constants): the host-side parameter stream."""

    MASK = (1 << 64) - 1

    def __init__(self, seed: int):
        self.state = seed & self.MASK

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & self.MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.MASK
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return ((self.next_u64() >> 11) + 0.5) * 2.0**-53

    def normal(self) -> float:
        u1, u2 = self.uniform(), self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


@dataclass
class Field:
    """One sensor's field: its kind, frame size, scalar parameters and (blobs) the blob table."""

    kind: int
    width: int
    height: int
    base: float = 0.0
    amp: float = 0.0
    nx: float = 0.0
    ny: float = 0.0
    c: float = 0.0
    speed: float = 0.0
    width_px: float = 1.0
    blobs: np.ndarray = field(default_factory=lambda: np.zeros((0, BLOB_WORDS), np.float32))

    @property
    def n_blobs(self) -> int:
        return int(self.blobs.shape[0])

    def scalars(self) -> np.ndarray:
        """The float32 scalar words in the order the C structs take them."""
        return np.array([self.base, self.amp, self.nx, self.ny, self.c, self.speed, self.width_px], np.float32)


def tanh_edge(width: int, height: int, seed: int, *, base=100.0, amp=80.0, speed=40.0, edge_px=1.5) -> Field:
    """E = base + amp tanh((n . p - speed t - c) / edge_px): n at a seed-uniform angle, c seed-uniform on
    [0, width] px."""
    g = SplitMix64(seed)
    phi = 2.0 * math.pi * g.uniform()
    c = width * g.uniform()
    f32 = lambda v: float(np.float32(v))  # noqa: E731
    return Field(KIND_TANH_EDGE, width, height, base=f32(base), amp=f32(amp), nx=f32(math.cos(phi)),
                 ny=f32(math.sin(phi)), c=f32(c), speed=f32(speed), width_px=f32(edge_px))


def blobs(width: int, height: int, seed: int, n_blobs: int, *, base=50.0, amp_mu=math.log(60.0), amp_sigma=0.5,
          r_lo=3.0, r_hi=20.0, v_sigma=60.0) -> Field:
    """base + sum of n_blobs Gaussian blobs: amplitude lognormal(amp_mu, amp_sigma), radius U[r_lo, r_hi] px,
    centre uniform on the array, constant velocity N(0, v_sigma) px/s per axis."""
    g = SplitMix64(seed)
    t = np.zeros((n_blobs, BLOB_WORDS), np.float32)
    for k in range(n_blobs):
        a = math.exp(amp_mu + amp_sigma * g.normal())
        r = r_lo + (r_hi - r_lo) * g.uniform()
        cx, cy = width * g.uniform(), height * g.uniform()
        vx, vy = v_sigma * g.normal(), v_sigma * g.normal()
        r32 = np.float32(r)
        t[k, 0] = a
        t[k, 1] = cx
        t[k, 2] = cy
        t[k, 3] = vx
        t[k, 4] = vy
        t[k, 5] = np.float32(1.0) / (np.float32(2.0) * r32 * r32)
        t[k, 6] = np.float32(36.0) * r32 * r32
        t[k, 7] = np.float32(9.0) * r32 * r32
        t[k, 8] = np.float32(math.hypot(float(np.float32(vx)), float(np.float32(vy))))
    return Field(KIND_BLOBS, width, height, base=float(np.float32(base)), blobs=t)
