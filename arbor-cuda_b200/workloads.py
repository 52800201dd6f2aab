"""Named workloads: camera/state records (C, 64 floats) and input records
(I, 32 floats) for the measured configurations.  Pure numpy; every
implementation (GPU library, CPU oracle, reference harness build) is fed the
same arrays.

Field maps follow the reference: C (Arbor.cu:179-182, 51, 277-304) and
I (Arbor.cu:182).
"""
from __future__ import annotations

import math

import numpy as np

FOREST_SEED = 7
TREE_SEED = 1


def hash_u(x: int) -> int:
    """The reference's integer hash (Arbor.cu:32)."""
    x &= 0xFFFFFFFF
    x ^= x >> 16
    x = (x * 2146121005) & 0xFFFFFFFF
    x ^= x >> 15
    x = (x * 2221713035) & 0xFFFFFFFF
    x ^= x >> 16
    return x


def rnd(n: int, seed: int) -> float:
    """Arbor.cu:33 - float32 value of the 24-bit hash fraction."""
    h = hash_u((n & 0xFFFFFFFF) ^ hash_u(seed & 0xFFFFFFFF))
    return float(np.float32(h & 16777215) / np.float32(16777216.0))


def forest_seed(tree: int, ws: int) -> int:
    """forestSeed (Arbor.cu:57): the per-tree seed of instance `tree` of world seed ws."""
    return hash_u((tree * 92821 + ws * 68917 + 17) & 0xFFFFFFFF) & 1048575


def forest_yaw(tree: int, ws: int) -> float:
    """forestYaw (Arbor.cu:66): rnd(4, forestSeed) * pi * 2 in float32."""
    return float(np.float32(np.float32(rnd(4, forest_seed(tree, ws))) * np.float32(3.14159265359)) * np.float32(2.0))


def species_of(n_species: int, ws: int = FOREST_SEED) -> np.ndarray:
    """Species of each of the 324 instances in a forest of n_species species:
    forestSeed(t, ws) mod n_species (a seeded, roughly even split)."""
    return np.array([forest_seed(t, ws) % n_species for t in range(324)], np.int32)


def base_state(seed: int, width: int, height: int) -> np.ndarray:
    """initCamera's defaults (Arbor.cu:181) without the pose."""
    C = np.zeros(64, np.float32)
    C[12] = -0.45
    C[13] = 0.63
    C[14] = 0.90
    C[20] = 1.18
    C[22] = 1.0
    C[23] = 1.0
    C[31] = seed
    C[44] = 1.0
    C[3] = 1.0
    C[18] = 1.0
    C[32] = width
    C[33] = height
    return C


def single_tree_camera(width: int = 256, height: int = 256, seed: int = TREE_SEED) -> np.ndarray:
    """One tree, first-person camera at 1.72 m eye height, 6 m from the
    trunk, 60 degree vertical field of view, looking at the crown centre
    (0, 5.4, 0); shadows off, lit view mode, first sample with history reset.

    cameraRay (Arbor.cu:51) spans v in [-0.5, 0.5] * C[14], so a 60 degree
    vertical FOV is C[14] = 2 tan(30 deg).
    """
    C = base_state(seed, width, height)
    C[0:3] = (0.0, 1.72, 6.0)
    C[4:7] = (0.0, 5.4, 0.0)
    C[14] = np.float32(2.0 * math.tan(math.radians(30.0)))
    C[16] = math.pi
    C[17] = math.atan2(5.4 - 1.72, 6.0)
    C[22] = 0.0
    C[15] = 0.0
    C[9] = 0.0
    C[10] = 1.0
    return C


def walk_input(frame: int, seed: int = FOREST_SEED) -> tuple[np.ndarray, float]:
    """Input record and dt of frame `frame` of the seeded forest walk.

    The walk uses the reference's own camera state machine (updateCamera,
    Arbor.cu:182): forward key held (I[15] = 1) and a mouse turn
    I[0] = (rnd(frame, seed) - 0.5) * 20 (a heading random walk of at most
    +-0.0225 rad per frame).  updateCamera walks at 4.2 m/s of `delta`, so
    delta = 1/180 s advances 4.2/180 m per frame: 1.4 m/s at 60 frames/s.
    Eye height is pinned to 1.72 m by updateCamera.
    """
    I = np.zeros(32, np.float32)
    I[0] = (rnd(frame, seed) - 0.5) * 20.0
    I[15] = 1.0
    return I, 1.0 / 180.0


def forest_start_state(width: int = 1920, height: int = 1080, seed: int = FOREST_SEED, shadows: bool = False) -> np.ndarray:
    """Walk start: initCamera's preset-1 pose (eye (2, 1.72, 18), yaw pi) is
    applied by running initCamera itself; this returns the fields the walk
    changes on top of it."""
    C = base_state(seed, width, height)
    C[22] = 1.0 if shadows else 0.0
    return C


def shadow_sun(seed: int = FOREST_SEED) -> tuple[float, float]:
    """Sun azimuth from the seed and 35 degree elevation (C[12], C[13])."""
    return 2.0 * math.pi * rnd(0, seed), math.radians(35.0)


VIEW_PRESETS = (1, 2, 3, 4, 5)


BATCH_RESOLUTIONS = ((320, 180), (640, 360), (1280, 720), (1920, 1080))


def batch_seeds(n: int, seed: int = FOREST_SEED) -> list[int]:
    """n master seeds: `seed` first, then seeds drawn from rnd(k, seed) over
    the engine's seed range 0..1,000,000 (src/engine.js:28)."""
    out = [seed]
    k = 1
    while len(out) < n:
        s = int(rnd(k, seed) * 1000000.0)
        if s not in out:
            out.append(s)
        k += 1
    return out


def view_pose_state(scene_seed: int, width: int, height: int, eye_x: float, eye_z: float, yaw: float, pitch: float,
                    shadows: bool = True) -> np.ndarray:
    """Camera/state record of a first-person view at (eye_x, 1.72, eye_z)
    looking along (yaw, pitch), as fpsPose lays it out (Arbor.cu:179): the
    look-at point is the eye plus the unit view direction; first sample with
    history reset; sun shadows at 35 degrees elevation, azimuth from the seed."""
    C = base_state(scene_seed, width, height)
    eye = np.array([eye_x, 1.72, eye_z], np.float64)
    f = np.array([math.sin(yaw) * math.cos(pitch), math.sin(pitch), math.cos(yaw) * math.cos(pitch)])
    C[0:3] = eye
    C[4:7] = eye + f
    C[16] = C[27] = yaw
    C[17] = C[28] = pitch
    C[22] = 1.0 if shadows else 0.0
    if shadows:
        C[12], C[13] = shadow_sun(scene_seed)
    C[9], C[10] = 0.0, 1.0
    return C


def batch_views(n_views: int, seeds: list[int], resolutions=BATCH_RESOLUTIONS, seed: int = FOREST_SEED, shadows: bool = True,
                extent: float = 200.0) -> list[tuple[int, int, int, np.ndarray]]:
    """(scene index, width, height, C) of n_views seeded views: resolution
    uniform over `resolutions`, scene uniform over the seeds, eye uniform in
    the forest square [-extent, extent]^2 at 1.72 m, yaw uniform, pitch
    uniform in [-0.05, 0.20] rad."""
    out = []
    for v in range(n_views):
        r = [rnd(1000 + 8 * v + k, seed) for k in range(6)]
        w, h = resolutions[min(int(r[0] * len(resolutions)), len(resolutions) - 1)]
        scene = min(int(r[1] * len(seeds)), len(seeds) - 1)
        C = view_pose_state(seeds[scene], w, h, (r[2] * 2.0 - 1.0) * extent, (r[3] * 2.0 - 1.0) * extent, r[4] * 2.0 * math.pi,
                            -0.05 + 0.25 * r[5], shadows)
        out.append((scene, w, h, C))
    return out
