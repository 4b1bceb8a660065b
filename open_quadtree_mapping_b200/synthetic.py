"""Seeded synthetic keyframes: a ray-cast textured box room.

The reference measures on a ROS bag that is not available offline; these
scenes stand in for it with the shapes and value ranges of the bench
configurations: 8-bit grayscale pinhole images, metric poses, and ground-truth
depth as the Euclidean distance to the surface point (the reference's output
convention, README.md:18-20).

Scene: a 10 x 6 x 4 m room (x length, y width, z up) holding 6 random
axis-aligned boxes.  Every face is textured by multi-octave value noise in
[0, 255] whose fine octaves are modulated by a slow "detail" field, so images
mix smooth regions (coarse quadtree levels) with fine texture.  Trajectories
move forward/laterally by 5-20 cm per frame with <= 3 degrees of rotation.
Camera frame: x right, y down, z forward; a pixel (u, v) samples the ray
through K^-1 [u, v, 1] (no half-pixel offset, matching
PinholeCamera::cam2world, camera_model/pinhole_camera.cuh:48-52).

Seeds follow the convention scene = 1000 + stream, trajectory = 2000 + stream.
"""
from __future__ import annotations

import dataclasses

import numpy as np

ROOM = np.array([10.0, 6.0, 4.0])


@dataclasses.dataclass
class Scene:
    boxes: np.ndarray  # (nb, 2, 3) lo/hi corners
    tex_seed: int


def make_scene(seed: int, n_boxes: int = 6) -> Scene:
    rng = np.random.default_rng(seed)
    boxes = []
    for _ in range(n_boxes):
        size = rng.uniform([0.4, 0.4, 0.4], [1.6, 1.6, 1.8])
        cx = rng.uniform(4.0, 9.2)
        cy = rng.uniform(0.6, 5.4)
        on_floor = rng.uniform() < 0.6
        z0 = 0.0 if on_floor else rng.uniform(0.3, 2.0)
        lo = np.array([cx - size[0] / 2, cy - size[1] / 2, z0])
        hi = np.minimum(lo + size, ROOM - 0.05)
        boxes.append((lo, hi))
    return Scene(np.array(boxes, dtype=np.float64), int(rng.integers(1, 2**31 - 1)))


def _hash01(ix, iy, salt):
    x = (ix.astype(np.int64) & 0xFFFFFFFF).astype(np.uint32) * np.uint32(0x8DA6B343)
    x ^= (iy.astype(np.int64) & 0xFFFFFFFF).astype(np.uint32) * np.uint32(0xD8163841)
    x ^= salt.astype(np.uint32) * np.uint32(0xCB1AB31F)
    x ^= x >> np.uint32(13)
    x *= np.uint32(0x5BD1E995)
    x ^= x >> np.uint32(15)
    return x.astype(np.float64) / 4294967296.0


def _value_noise(s, t, salt):
    i0 = np.floor(s)
    j0 = np.floor(t)
    fs = s - i0
    ft = t - j0
    ws = fs * fs * (3 - 2 * fs)
    wt = ft * ft * (3 - 2 * ft)
    i0 = i0.astype(np.int64)
    j0 = j0.astype(np.int64)
    v00 = _hash01(i0, j0, salt)
    v10 = _hash01(i0 + 1, j0, salt)
    v01 = _hash01(i0, j0 + 1, salt)
    v11 = _hash01(i0 + 1, j0 + 1, salt)
    a = v00 + (v10 - v00) * ws
    b = v01 + (v11 - v01) * ws
    return a + (b - a) * wt


def _texture(s, t, surf, tex_seed):
    salt0 = (surf.astype(np.int64) * 7919 + tex_seed) & 0x7FFFFFFF
    detail = _value_noise(s * 0.45 + 11.3, t * 0.45 - 3.1, salt0 + 1)
    detail = np.clip((detail - 0.35) * 2.5, 0.0, 1.0)
    val = np.zeros_like(s)
    amp_sum = 0.0
    freq = 1.3
    for k in range(6):
        amp = 0.55**k
        a = amp * (1.0 if k < 2 else detail)
        val += a * _value_noise(s * freq + 0.37 * k, t * freq - 0.71 * k, salt0 + 17 * (k + 2))
        amp_sum += amp
        freq *= 2.1
    val = val / amp_sum
    base = _hash01(surf.astype(np.int64), surf.astype(np.int64) * 3, salt0 * 0 + tex_seed)
    val = 0.5 + 1.6 * (val - 0.5) + 0.25 * (base - 0.5)
    return np.clip(val, 0.0, 1.0)


def render(scene: Scene, T_world_cam: np.ndarray, W: int, H: int, fx: float, fy: float,
           cx: float, cy: float):
    """Ray-casts one view. Returns (u8 image HxW, float32 Euclidean depth HxW)."""
    u, v = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))
    u = u.ravel()
    v = v.ravel()
    dcx = (u - cx) / fx
    dcy = (v - cy) / fy
    nrm = 1.0 / np.sqrt(dcx * dcx + dcy * dcy + 1.0)
    dcx *= nrm
    dcy *= nrm
    R = T_world_cam[:3, :3]
    o = T_world_cam[:3, 3]
    d = [R[k, 0] * dcx + R[k, 1] * dcy + R[k, 2] * nrm for k in range(3)]
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = [1.0 / d[k] for k in range(3)]
        # room interior: exit distance along each axis, nearest exit wins
        t_best = None
        for k in range(3):
            tl = (0.0 - o[k]) * inv[k]
            th = (ROOM[k] - o[k]) * inv[k]
            tk = np.maximum(tl, th)
            sk = (th >= tl).astype(np.int64)
            if t_best is None:
                t_best, axis, surf = tk, np.zeros(tk.shape, np.int64), sk
            else:
                better = tk < t_best
                t_best = np.where(better, tk, t_best)
                axis = np.where(better, k, axis)
                surf = np.where(better, 2 * k + sk, surf)
        for b, (lo, hi) in enumerate(scene.boxes):
            tn = tf = None
            for k in range(3):
                t1 = (lo[k] - o[k]) * inv[k]
                t2 = (hi[k] - o[k]) * inv[k]
                tmin = np.minimum(t1, t2)
                tmax = np.maximum(t1, t2)
                sd = (t1 > t2).astype(np.int64)
                if tn is None:
                    tn, tf, ax, side = tmin, tmax, np.zeros(tmin.shape, np.int64), sd
                else:
                    bigger = tmin > tn
                    tn = np.where(bigger, tmin, tn)
                    ax = np.where(bigger, k, ax)
                    side = np.where(bigger, sd, side)
                    tf = np.minimum(tf, tmax)
            hit = (tn <= tf) & (tn > 1e-6) & (tn < t_best)
            t_best = np.where(hit, tn, t_best)
            surf = np.where(hit, 6 + b * 6 + ax * 2 + side, surf)
            axis = np.where(hit, ax, axis)
    P = [o[k] + d[k] * t_best for k in range(3)]
    # texture coordinates: the two world axes spanning the face
    s = np.where(axis == 0, P[1], P[0])
    t = np.where(axis == 2, P[1], P[2])
    val = _texture(s * 3.0, t * 3.0, surf, scene.tex_seed)
    img = np.clip(np.round(val * 255.0), 0, 255).astype(np.uint8).reshape(H, W)
    depth = t_best.reshape(H, W).astype(np.float32)
    return img, depth


def _rot(axis: int, ang: float):
    c, s = np.cos(ang), np.sin(ang)
    R = np.eye(3)
    i, j = [(1, 2), (0, 2), (0, 1)][axis]
    R[i, i] = c
    R[j, j] = c
    R[i, j] = -s
    R[j, i] = s
    return R


def make_trajectory(seed: int, n: int):
    """n camera-to-world poses (4x4, float64) along a forward/lateral path."""
    rng = np.random.default_rng(seed)
    # camera looking along world +x, right = -y, down = -z
    R0 = np.array([[0.0, 0.0, 1.0], [-1.0, 0.0, 0.0], [0.0, -1.0, 0.0]])
    yaw = rng.uniform(-0.25, 0.25)
    R = _rot(2, yaw) @ R0
    pos = np.array([rng.uniform(1.2, 2.2), rng.uniform(2.2, 3.8), rng.uniform(1.2, 2.0)])
    poses = []
    for _ in range(n):
        T = np.eye(4)
        T[:3, :3] = R
        T[:3, 3] = pos
        poses.append(T)
        base = rng.uniform(0.05, 0.20)
        heading = rng.uniform(-0.9, 0.9)  # mix of forward and lateral motion (radians)
        fwd = R[:, 2]
        right = R[:, 0]
        step = np.cos(heading) * fwd + np.sin(heading) * right
        step[2] *= 0.3
        step /= np.linalg.norm(step)
        pos = pos + base * step
        dR = (_rot(0, rng.uniform(-1, 1) * np.deg2rad(1.7))
              @ _rot(1, rng.uniform(-1, 1) * np.deg2rad(1.7))
              @ _rot(2, rng.uniform(-1, 1) * np.deg2rad(1.0)))
        R = R @ dR
    return poses


def inv_se3(T):
    Ti = np.eye(4)
    Ti[:3, :3] = T[:3, :3].T
    Ti[:3, 3] = -T[:3, :3].T @ T[:3, 3]
    return Ti


@dataclasses.dataclass
class Keyframe:
    """One reference image with its measurement frames.

    T_meas_ref[f] is the 3x4 row-major float32 transform taking points from
    the reference camera into measurement frame f (the reference's
    FrameElement::transform as built in seed_matrix.cu:457-464).
    """
    W: int
    H: int
    fx: float
    fy: float
    cx: float
    cy: float
    ref: np.ndarray          # (H, W) u8
    gt_depth: np.ndarray     # (H, W) f32 Euclidean depth
    meas: np.ndarray         # (F, H, W) u8, most recent first
    T_meas_ref: np.ndarray   # (F, 12) f32
    T_world_ref: np.ndarray  # (4, 4) f64
    T_world_meas: np.ndarray # (F, 4, 4) f64


def make_keyframe(stream: int, W=752, H=480, fx=460.0, fy=460.0, cx=None, cy=None,
                  F=5) -> Keyframe:
    cx = W / 2.0 if cx is None else cx
    cy = H / 2.0 if cy is None else cy
    scene = make_scene(1000 + stream)
    traj = make_trajectory(2000 + stream, F + 1)
    T_ref = traj[F]
    ref, gt = render(scene, T_ref, W, H, fx, fy, cx, cy)
    meas, Ts, Tw = [], [], []
    for k in range(F):
        Tm = traj[F - 1 - k]  # most recent first
        img, _ = render(scene, Tm, W, H, fx, fy, cx, cy)
        meas.append(img)
        Tw.append(Tm)
        Ts.append((inv_se3(Tm) @ T_ref)[:3, :4].reshape(-1))
    return Keyframe(W, H, float(fx), float(fy), float(cx), float(cy), ref, gt,
                    np.stack(meas), np.array(Ts, dtype=np.float32), T_ref, np.stack(Tw))


def make_sequence(stream: int, n: int, W=752, H=480, fx=460.0, fy=460.0, cx=None, cy=None):
    """n consecutive frames of one stream: (u8 images (n,H,W), T_curr_world (n,12) f32,
    gt depth (n,H,W) f32).  T_curr_world is the world-to-camera transform the
    Depthmap facade takes (depthmap.h:46-47)."""
    cx = W / 2.0 if cx is None else cx
    cy = H / 2.0 if cy is None else cy
    scene = make_scene(1000 + stream)
    traj = make_trajectory(2000 + stream, n)
    imgs, Ts, gts = [], [], []
    for T in traj:
        img, gt = render(scene, T, W, H, fx, fy, cx, cy)
        imgs.append(img)
        gts.append(gt)
        Ts.append(inv_se3(T)[:3, :4].reshape(-1))
    return np.stack(imgs), np.array(Ts, dtype=np.float32), np.stack(gts)


def render_frame(args):
    """(scene seed, T_world_cam, W, H, f) -> u8 image with the principal point
    at the image centre; a picklable job for process pools."""
    seed, T, W, H, f = args
    img, _ = render(make_scene(seed), T, W, H, f, f, W / 2.0, H / 2.0)
    return img
