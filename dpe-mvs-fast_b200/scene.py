"""Seeded synthetic multi-view scenes in the reference's input formats.

The reference is run on ETH3D scenes (images/, cams/, pair.txt; RUN_MVS_EXP.md:19-36), which are
not available here.  This module ray-casts stand-in scenes with the shapes, sizes and value
distributions of the measured workloads: planes and spheres textured with 3-D value noise, seen by
pinhole cameras on an arc looking at the origin.  It returns images, cameras, ground-truth depth
and normals, and can write a dense folder in the reference formats:

* ``cams/%08d_cam.txt``  -- ``extrinsic`` 4x4, ``intrinsic`` 3x3, ``dmin interval num dmax``
  (read by ReadCamera, DPE.cpp:341-382),
* ``pair.txt``           -- view count, then per view its id and ``n id score ...``
  (read by GenerateSampleList, main.cpp:102-145),
* ``images/%08d.jpg``    -- 8-bit images (decoded by cv2 when available).

Everything is computed with torch on the requested device (CPU for tests, CUDA for the bench
setup); the generator is deterministic for a given seed and device.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional

import numpy as np
import torch


@dataclasses.dataclass
class SceneSpec:
    width: int = 640
    height: int = 480
    n_views: int = 5
    fx: float = 525.0
    fy: float = 525.0
    cx: float = 320.0
    cy: float = 240.0
    arc_radius: float = 2.0
    step_deg: float = 10.0
    n_planes: int = 3
    n_spheres: int = 1
    tex_mean: float = 128.0
    tex_sigma: float = 40.0          # strong-texture noise sigma (grey levels)
    weak_sigma: Optional[float] = None  # when set, about half of the objects use this sigma
    weak_sigma_range: Optional[tuple] = None  # per-object sigma drawn from this range instead
    image_noise: float = 0.0         # additive Gaussian pixel noise (grey levels)
    depth_min: float = 1.5
    depth_max: float = 3.0
    tex_freq: float = 25.0           # base noise frequency, cycles per metre
    supersample: int = 2
    ring: bool = False               # cameras on a full circle (360 / n_views apart) instead of an arc
    wall_radius: Optional[float] = None  # ring scenes: a textured cylinder wall around the objects


def preset(name: str) -> SceneSpec:
    """Named workloads.  c1..c3 follow the measured configurations; 'tiny'/'small' are test sizes."""
    if name == "c1":   # 5 views 640x480, 3 planes + 1 sphere, sigma 40
        return SceneSpec()
    if name == "c2":   # 10 views 1600x1200, 6 planes + 2 spheres, half the area sigma 3
        return SceneSpec(width=1600, height=1200, n_views=10, fx=1312.5, fy=1312.5, cx=800.0, cy=600.0,
                         n_planes=6, n_spheres=2, weak_sigma=3.0, tex_freq=60.0, supersample=1)
    if name == "c3":   # 10 views 1920x1080, mean 200, sigma 2-8, +N(0,1)
        return SceneSpec(width=1920, height=1080, n_views=10, fx=1575.0, fy=1575.0, cx=960.0, cy=540.0,
                         n_planes=6, n_spheres=2, tex_mean=200.0, weak_sigma_range=(2.0, 8.0),
                         image_noise=1.0, tex_freq=60.0, supersample=1)
    if name == "tiny":  # 3 views 64x48
        return SceneSpec(width=64, height=48, n_views=3, fx=52.5, fy=52.5, cx=32.0, cy=24.0, tex_freq=2.5)
    if name == "small":  # 4 views 160x120
        return SceneSpec(width=160, height=120, n_views=4, fx=131.25, fy=131.25, cx=80.0, cy=60.0, tex_freq=6.0)
    if name == "small_weak":  # 4 views 192x144 with near-textureless objects (~20% WEAK pixels)
        return SceneSpec(width=192, height=144, n_views=4, fx=157.5, fy=157.5, cx=96.0, cy=72.0,
                         n_planes=4, n_spheres=1, weak_sigma=1.0, image_noise=0.7, tex_freq=7.5)
    if name == "c2_small":  # the c2 scene layout at 400x300 (coarse pyramid level)
        return SceneSpec(width=400, height=300, n_views=10, fx=328.125, fy=328.125, cx=200.0, cy=150.0,
                         n_planes=6, n_spheres=2, weak_sigma=3.0, tex_freq=15.0, supersample=1)
    if name == "c2_200":  # the c2 scene layout at 200x150 (the CPU reference's timing sample)
        return SceneSpec(width=200, height=150, n_views=10, fx=164.0625, fy=164.0625, cx=100.0, cy=75.0,
                         n_planes=6, n_spheres=2, weak_sigma=3.0, tex_freq=7.5, supersample=1)
    if name == "c5_ring":  # 60 cameras on a ring around 5 planes + 3 spheres inside a textured wall;
        # intrinsics at 640x480, scaled for the 1600x1200 and 3200x2400 renderings (camera_struct)
        return SceneSpec(width=640, height=480, n_views=60, fx=525.0, fy=525.0, cx=320.0, cy=240.0,
                         arc_radius=2.0, n_planes=6, n_spheres=3, tex_sigma=40.0, depth_min=1.0, depth_max=5.2,
                         tex_freq=40.0, supersample=1, ring=True, wall_radius=3.0)
    raise ValueError(f"unknown scene preset {name!r}")


@dataclasses.dataclass
class Scene:
    spec: SceneSpec
    K: np.ndarray            # (N, 3, 3) float32
    R: np.ndarray            # (N, 3, 3) float32 world -> camera rotation
    t: np.ndarray            # (N, 3) float32
    gray: np.ndarray         # (N, H, W) uint8
    bgr: np.ndarray          # (N, H, W, 3) uint8
    depth: np.ndarray        # (N, H, W) float32 ground truth (z in camera)
    normal: np.ndarray       # (N, H, W, 3) float32 ground-truth world normals
    pairs: List[List[int]]   # per view: source ids, best first
    scores: List[List[float]]

    @property
    def n(self) -> int:
        return self.gray.shape[0]


def _hash3(i, j, k, seed: int):
    m = 0xFFFFFFFF
    h = (i * 73856093) ^ (j * 19349663) ^ (k * 83492791) ^ seed
    h = h & m
    h = ((h ^ (h >> 16)) * 0x45D9F3B) & m
    h = ((h ^ (h >> 16)) * 0x45D9F3B) & m
    h = h ^ (h >> 16)
    return h.to(torch.float32) * (2.0 / 4294967296.0) - 1.0


def _value_noise(p: torch.Tensor, seed: int) -> torch.Tensor:
    """Trilinear value noise with smoothstep weights at points p (M, 3)."""
    f = torch.floor(p)
    w = p - f
    w = w * w * (3.0 - 2.0 * w)
    i = f.to(torch.int64)
    out = torch.zeros(p.shape[0], dtype=torch.float32, device=p.device)
    for dx in (0, 1):
        wx = w[:, 0] if dx else 1.0 - w[:, 0]
        for dy in (0, 1):
            wy = w[:, 1] if dy else 1.0 - w[:, 1]
            for dz in (0, 1):
                wz = w[:, 2] if dz else 1.0 - w[:, 2]
                out += wx * wy * wz * _hash3(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
    return out


def _texture(p: torch.Tensor, seed: int, freq: float) -> torch.Tensor:
    """4-octave value noise, roughly zero mean and unit variance."""
    acc = torch.zeros(p.shape[0], dtype=torch.float32, device=p.device)
    amp, norm = 1.0, 0.0
    for o in range(4):
        acc += amp * _value_noise(p * (freq * (2.0 ** o)), seed + 7919 * o)
        norm += amp * amp
        amp *= 0.5
    # a single value-noise octave has a standard deviation of about 0.36 (uniform lattice, smoothstep)
    return acc / (math.sqrt(norm) * 0.36)


def _intersect(objs, C: torch.Tensor, dw: torch.Tensor, dev):
    """Nearest hit of the rays C + t dw (dw: (M, 3)) with the objects: (t, object index, normal);
    t = inf and index -1 where nothing is hit."""
    f32 = torch.float32
    M = dw.shape[0]
    best_t = torch.full((M,), float("inf"), device=dev)
    best_o = torch.full((M,), -1, dtype=torch.int64, device=dev)
    best_n = torch.zeros(M, 3, device=dev)
    for oi, ob in enumerate(objs):
        if ob["kind"] == "plane":
            n = torch.tensor(ob["n"], dtype=f32, device=dev)
            c = torch.tensor(ob["c"], dtype=f32, device=dev)
            den = dw @ n
            tt = ((c - C) @ n) / den
            P = C + tt[:, None] * dw
            rel = P - c
            uu = rel @ torch.tensor(ob["u"], dtype=f32, device=dev)
            vv = rel @ torch.tensor(ob["v"], dtype=f32, device=dev)
            ok = (tt > 0) & (uu.abs() <= ob["hu"]) & (vv.abs() <= ob["hv"])
            nn = n.expand(M, 3)
        elif ob["kind"] == "sphere":
            c = torch.tensor(ob["c"], dtype=f32, device=dev)
            oc = C - c
            a = (dw * dw).sum(1)
            b = 2.0 * (dw @ oc)
            cc = float(oc @ oc - ob["r"] ** 2)
            disc = b * b - 4 * a * cc
            ok = disc > 0
            tt = (-b - torch.sqrt(disc.clamp_min(0))) / (2 * a)
            ok = ok & (tt > 0)
            P = C + tt[:, None] * dw
            nn = (P - c) / ob["r"]
        else:  # "wall": the inside of a vertical (y) cylinder of radius r around the origin
            a = dw[:, 0] * dw[:, 0] + dw[:, 2] * dw[:, 2]
            b = 2.0 * (C[0] * dw[:, 0] + C[2] * dw[:, 2])
            cc = float(C[0] * C[0] + C[2] * C[2] - ob["r"] ** 2)
            disc = b * b - 4 * a * cc
            tt = (-b + torch.sqrt(disc.clamp_min(0))) / (2 * a)
            ok = (disc > 0) & (tt > 0)
            P = C + tt[:, None] * dw
            nn = torch.stack([-P[:, 0], torch.zeros_like(P[:, 0]), -P[:, 2]], 1) / ob["r"]
        upd = ok & (tt < best_t)
        best_t = torch.where(upd, tt, best_t)
        best_o = torch.where(upd, torch.full_like(best_o, oi), best_o)
        best_n = torch.where(upd[:, None], nn, best_n)
    return best_t, best_o, best_n


def _look_at_camera(theta: float, radius: float):
    C = np.array([radius * math.sin(theta), 0.0, -radius * math.cos(theta)])
    z = -C / np.linalg.norm(C)
    y_down = np.array([0.0, 1.0, 0.0])
    x = np.cross(y_down, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    R = np.stack([x, y, z])
    t = -R @ C
    return R, t


def make_scene(spec: SceneSpec | str, seed: int = 1, device: str = "cpu") -> Scene:
    if isinstance(spec, str):
        spec = preset(spec)
    rng = np.random.default_rng(seed)
    N, H, W = spec.n_views, spec.height, spec.width
    K = np.array([[spec.fx, 0, spec.cx], [0, spec.fy, spec.cy], [0, 0, 1]], dtype=np.float64)
    Rs, ts = [], []
    for v in range(N):
        theta = math.radians((v - (N - 1) / 2.0) * spec.step_deg)
        R, t = _look_at_camera(theta, spec.arc_radius)
        Rs.append(R)
        ts.append(t)

    # ---- objects: a far background plane, n_planes-1 tilted rectangles, spheres
    objs = []
    span = 0.5 * (spec.depth_max - spec.depth_min)
    mid = spec.depth_min + span - spec.arc_radius  # object-centre offset along +z from the origin
    objs.append(dict(kind="plane", c=np.array([0.0, 0.0, spec.depth_max - spec.arc_radius - 0.45 * span]),
                     n=np.array([0.0, 0.0, -1.0]), u=np.array([1.0, 0, 0]), v=np.array([0, 1.0, 0]),
                     hu=1e3, hv=1e3))
    for _ in range(spec.n_planes - 1):
        c = np.array([rng.uniform(-0.35, 0.35), rng.uniform(-0.25, 0.25), mid + rng.uniform(-0.6, 0.4) * span])
        tilt = rng.uniform(-0.6, 0.6, size=2)
        n = np.array([math.sin(tilt[0]), math.sin(tilt[1]), -1.0])
        n /= np.linalg.norm(n)
        u = np.cross(np.array([0.0, 1.0, 0.0]), n)
        u /= np.linalg.norm(u)
        vv = np.cross(n, u)
        objs.append(dict(kind="plane", c=c, n=n, u=u, v=vv, hu=rng.uniform(0.12, 0.3), hv=rng.uniform(0.1, 0.25)))
    for _ in range(spec.n_spheres):
        c = np.array([rng.uniform(-0.3, 0.3), rng.uniform(-0.2, 0.2), mid + rng.uniform(-0.5, 0.1) * span])
        objs.append(dict(kind="sphere", c=c, r=rng.uniform(0.08, 0.18)))
    n_obj = len(objs)
    sigmas = np.full(n_obj, spec.tex_sigma)
    if spec.weak_sigma is not None:
        # about half of the visible area: the background plus every other foreground object
        sigmas[0] = spec.weak_sigma
        sigmas[2::2] = spec.weak_sigma
    if spec.weak_sigma_range is not None:
        sigmas = rng.uniform(spec.weak_sigma_range[0], spec.weak_sigma_range[1], size=n_obj)
    tints = rng.uniform(0.85, 1.15, size=(n_obj, 3))
    tex_seed = int(rng.integers(1, 2**31 - 1))
    noise_seed = int(rng.integers(1, 2**31 - 1))

    dev = torch.device(device)
    f32 = torch.float32
    gray = np.zeros((N, H, W), np.uint8)
    bgr = np.zeros((N, H, W, 3), np.uint8)
    depth = np.zeros((N, H, W), np.float32)
    normal = np.zeros((N, H, W, 3), np.float32)
    ss = max(1, spec.supersample)
    offs = [((a + 0.5) / ss - 0.5, (b + 0.5) / ss - 0.5) for a in range(ss) for b in range(ss)]
    Kinv = torch.tensor(np.linalg.inv(K), dtype=f32, device=dev)
    vs, us = torch.meshgrid(torch.arange(H, device=dev, dtype=f32), torch.arange(W, device=dev, dtype=f32), indexing="ij")
    for v in range(N):
        R = torch.tensor(Rs[v], dtype=f32, device=dev)
        C = torch.tensor(-Rs[v].T @ ts[v], dtype=f32, device=dev)
        acc_val = torch.zeros(H * W, dtype=f32, device=dev)
        acc_col = torch.zeros(H * W, 3, dtype=f32, device=dev)
        for si, (ox, oy) in enumerate(offs):
            pix = torch.stack([(us + ox).reshape(-1), (vs + oy).reshape(-1), torch.ones(H * W, device=dev)], 1)
            dcam = pix @ Kinv.T
            dw = dcam @ R  # R^T * dcam
            best_t, best_o, best_n = _intersect(objs, C, dw, dev)
            P = C + best_t[:, None] * dw
            tex = _texture(P, tex_seed, spec.tex_freq)
            sig = torch.tensor(sigmas, dtype=f32, device=dev)[best_o.clamp_min(0)]
            val = spec.tex_mean + sig * tex
            acc_val += val
            acc_col += val[:, None] * torch.tensor(tints, dtype=f32, device=dev)[best_o.clamp_min(0)]
            if si == 0 or ss == 1:
                z = (P - C) @ R[2]
                # ground truth at the pixel centre: the first sample when ss == 1, else recast below
            if ss == 1:
                gt_z, gt_n = z, best_n
        if ss > 1:
            # ground truth at the exact pixel centre
            pix = torch.stack([us.reshape(-1), vs.reshape(-1), torch.ones(H * W, device=dev)], 1)
            dw = (pix @ Kinv.T) @ R
            best_t, _, best_n = _intersect(objs, C, dw, dev)
            gt_z = ((C + best_t[:, None] * dw) - C) @ R[2]
            gt_n = best_n
        val = acc_val / len(offs)
        col = acc_col / len(offs)
        if spec.image_noise > 0:
            g = torch.Generator(device=dev)
            g.manual_seed(noise_seed + v)
            val = val + spec.image_noise * torch.randn(val.shape, generator=g, device=dev)
            col = col + spec.image_noise * torch.randn(col.shape, generator=g, device=dev)
        gray[v] = torch.round(val.clamp(0, 255)).to(torch.uint8).reshape(H, W).cpu().numpy()
        bgr[v] = torch.round(col.clamp(0, 255)).to(torch.uint8).reshape(H, W, 3).cpu().numpy()
        depth[v] = gt_z.reshape(H, W).cpu().numpy()
        # orient normals towards the camera
        nrm = gt_n
        facing = ((C - (C + best_t[:, None] * dw if ss > 1 else P)) * nrm).sum(1) < 0
        nrm = torch.where(facing[:, None], -nrm, nrm)
        normal[v] = nrm.reshape(H, W, 3).cpu().numpy()

    pairs, scores = [], []
    for v in range(N):
        others = sorted((o for o in range(N) if o != v), key=lambda o: (abs(o - v), o))[:20]
        pairs.append(others)
        scores.append([round(100.0 / (1 + abs(o - v)), 3) for o in others])
    Kf = np.repeat(K[None].astype(np.float32), N, 0)
    return Scene(spec=spec, K=Kf, R=np.stack(Rs).astype(np.float32), t=np.stack(ts).astype(np.float32),
                 gray=gray, bgr=bgr, depth=depth, normal=normal, pairs=pairs, scores=scores)


def camera_struct(scene: Scene, v: int, width: int | None = None, height: int | None = None) -> dict:
    """A camera in the reference layout (ReadCamera + SceneCache::GetCamera scaling, DPE.cpp:739-760)."""
    K = scene.K[v].astype(np.float32).copy()
    W0, H0 = scene.spec.width, scene.spec.height
    width = W0 if width is None else width
    height = H0 if height is None else height
    sx = np.float32(width) / np.float32(W0)
    sy = np.float32(height) / np.float32(H0)
    K[0, 0] *= sx
    K[0, 2] *= sx
    K[1, 1] *= sy
    K[1, 2] *= sy
    R = scene.R[v].astype(np.float32)
    t = scene.t[v].astype(np.float32)
    # camera centre computed in double, as ReadCamera does (DPE.cpp:366-369)
    c = np.array([-(float(R[0, j]) * float(t[0]) + float(R[1, j]) * float(t[1]) + float(R[2, j]) * float(t[2]))
                  for j in range(3)], dtype=np.float32)
    return dict(K=K.reshape(-1), R=R.reshape(-1), t=t, c=c, height=height, width=width,
                depth_min=np.float32(scene.spec.depth_min), depth_max=np.float32(scene.spec.depth_max))


def write_dense_folder(scene: Scene, folder: str) -> None:
    """images/%08d.jpg, cams/%08d_cam.txt and pair.txt in the reference formats."""
    os.makedirs(os.path.join(folder, "images"), exist_ok=True)
    os.makedirs(os.path.join(folder, "cams"), exist_ok=True)
    try:
        import cv2
    except ImportError:  # pragma: no cover
        cv2 = None
    for v in range(scene.n):
        if cv2 is not None:
            cv2.imwrite(os.path.join(folder, "images", f"{v:08d}.jpg"), scene.bgr[v], [cv2.IMWRITE_JPEG_QUALITY, 100])
        R, t, K = scene.R[v], scene.t[v], scene.K[v]
        with open(os.path.join(folder, "cams", f"{v:08d}_cam.txt"), "w") as f:
            f.write("extrinsic\n")
            for i in range(3):
                f.write(f"{R[i,0]:.9g} {R[i,1]:.9g} {R[i,2]:.9g} {t[i]:.9g}\n")
            f.write("0 0 0 1\n\nintrinsic\n")
            for i in range(3):
                f.write(f"{K[i,0]:.9g} {K[i,1]:.9g} {K[i,2]:.9g}\n")
            d0, d1 = scene.spec.depth_min, scene.spec.depth_max
            f.write(f"\n{d0:.9g} {(d1 - d0) / 192:.9g} 192 {d1:.9g}\n")
    with open(os.path.join(folder, "pair.txt"), "w") as f:
        f.write(f"{scene.n}\n")
        for v in range(scene.n):
            f.write(f"{v}\n{len(scene.pairs[v])} " + " ".join(f"{o} {s}" for o, s in zip(scene.pairs[v], scene.scores[v])) + "\n")


# ---------------------------------------------------------------------------- ring scenes (C5)
class RingScene:
    """Cameras on a full ring around a cluster of planes and spheres inside a textured cylinder wall,
    rendered on demand at any resolution: the intrinsics of the spec (at spec.width x spec.height)
    are scaled as camera_struct scales them, so a rendering and its camera struct agree."""

    def __init__(self, spec: SceneSpec | str, seed: int = 1, device: str = "cpu"):
        if isinstance(spec, str):
            spec = preset(spec)
        assert spec.ring and spec.wall_radius, "a ring spec with a wall"
        self.spec, self.device = spec, device
        rng = np.random.default_rng(seed)
        N = spec.n_views
        self.R, self.t = [], []
        for v in range(N):
            R, t = _look_at_camera(2.0 * math.pi * v / N, spec.arc_radius)
            self.R.append(R.astype(np.float32))
            self.t.append(t.astype(np.float32))
        objs = [dict(kind="wall", r=spec.wall_radius)]
        for _ in range(spec.n_planes - 1):
            c = np.array([rng.uniform(-0.5, 0.5), rng.uniform(-0.3, 0.3), rng.uniform(-0.5, 0.5)])
            n = rng.normal(size=3)
            n /= np.linalg.norm(n)
            u = np.cross(np.array([0.0, 1.0, 0.0]) if abs(n[1]) < 0.9 else np.array([1.0, 0.0, 0.0]), n)
            u /= np.linalg.norm(u)
            objs.append(dict(kind="plane", c=c, n=n, u=u, v=np.cross(n, u), hu=rng.uniform(0.15, 0.35),
                             hv=rng.uniform(0.12, 0.3)))
        for _ in range(spec.n_spheres):
            c = np.array([rng.uniform(-0.45, 0.45), rng.uniform(-0.25, 0.25), rng.uniform(-0.45, 0.45)])
            objs.append(dict(kind="sphere", c=c, r=rng.uniform(0.1, 0.25)))
        self.objs = objs
        self.sigmas = np.full(len(objs), spec.tex_sigma)
        self.tints = rng.uniform(0.85, 1.15, size=(len(objs), 3))
        self.tex_seed = int(rng.integers(1, 2**31 - 1))
        self._K0 = np.array([[spec.fx, 0, spec.cx], [0, spec.fy, spec.cy], [0, 0, 1]], dtype=np.float32)

    @property
    def n(self) -> int:
        return self.spec.n_views

    def camera(self, v: int, width: int, height: int) -> dict:
        """camera_struct of ring camera v at width x height."""
        shim = Scene(spec=self.spec, K=self._K0[None].repeat(self.n, 0), R=np.stack(self.R), t=np.stack(self.t),
                     gray=np.zeros((0, 1, 1), np.uint8), bgr=None, depth=None, normal=None, pairs=[], scores=[])
        return camera_struct(shim, v, width, height)

    def render(self, v: int, width: int, height: int):
        """(gray uint8 HxW, bgr uint8 HxWx3, depth float32 HxW) of ring camera v, one ray per pixel
        centre."""
        dev = torch.device(self.device)
        f32 = torch.float32
        cam = self.camera(v, width, height)
        K = np.asarray(cam["K"], np.float64).reshape(3, 3)
        Kinv = torch.tensor(np.linalg.inv(K), dtype=f32, device=dev)
        R = torch.tensor(self.R[v], dtype=f32, device=dev)
        C = torch.tensor(-self.R[v].astype(np.float64).T @ self.t[v].astype(np.float64), dtype=f32, device=dev)
        H, W = height, width
        vs, us = torch.meshgrid(torch.arange(H, device=dev, dtype=f32), torch.arange(W, device=dev, dtype=f32), indexing="ij")
        pix = torch.stack([us.reshape(-1), vs.reshape(-1), torch.ones(H * W, device=dev)], 1)
        dw = (pix @ Kinv.T) @ R
        del pix, vs, us
        best_t, best_o, _ = _intersect(self.objs, C, dw, dev)
        P = C + best_t[:, None] * dw
        del dw
        tex = _texture(P, self.tex_seed, self.spec.tex_freq)
        o = best_o.clamp_min(0)
        val = self.spec.tex_mean + torch.tensor(self.sigmas, dtype=f32, device=dev)[o] * tex
        col = val[:, None] * torch.tensor(self.tints, dtype=f32, device=dev)[o]
        z = (P - C) @ R[2]
        gray = torch.round(val.clamp(0, 255)).to(torch.uint8).reshape(H, W).cpu().numpy()
        bgr = torch.round(col.clamp(0, 255)).to(torch.uint8).reshape(H, W, 3).cpu().numpy()
        return gray, bgr, z.reshape(H, W).cpu().numpy().astype(np.float32)


# The batching workload: 49 reference views of uneven resolution on the 60-camera ring, each with
# its 10 nearest ring neighbours as sources (rendered at the reference view's resolution).
C5_CLASSES = ((640, 480, 20), (1600, 1200, 20), (3200, 2400, 9))


def c5_views(n_ring: int = 60):
    """[(reference camera, width, height, [10 source cameras])] of the batching workload: the
    references spread over the ring, class by class; sources nearest first."""
    out = []
    total = sum(c[2] for c in C5_CLASSES)
    refs = [int(round(i * n_ring / total)) % n_ring for i in range(total)]
    k = 0
    for W, H, count in C5_CLASSES:
        for _ in range(count):
            r = refs[k]
            k += 1
            srcs = sorted(((r + d) % n_ring for d in (-1, 1, -2, 2, -3, 3, -4, 4, -5, 5)),
                          key=lambda o: (min((o - r) % n_ring, (r - o) % n_ring), o))
            out.append((r, W, H, srcs))
    return out


def c5_workload(seed: int = 1, device: str = "cpu", views=None):
    """The 49 per-view problems of the batching workload: per reference view its images (reference
    first, float32), cameras, ground-truth depth and colour.  `views` restricts it to a subset of
    c5_views() (indices).  Each rendering is kept only until the last problem that uses it."""
    ring = RingScene("c5_ring", seed=seed, device=device)
    layout = c5_views(ring.n)
    if views is not None:
        layout = [layout[i] for i in views]
    last = {}  # rendering -> index of the last problem that uses it
    for i, (r, W, H, srcs) in enumerate(layout):
        for v in [r] + srcs:
            last[(v, W, H)] = i
    cache = {}
    problems = []
    for i, (r, W, H, srcs) in enumerate(layout):
        imgs, cams = [], []
        for v in [r] + srcs:
            key = (v, W, H)
            if key not in cache:
                cache[key] = ring.render(v, W, H)
            imgs.append(cache[key][0].astype(np.float32))
            cams.append(ring.camera(v, W, H))
        _, bgr, z = cache[(r, W, H)]
        problems.append(dict(ref=r, width=W, height=H, sources=srcs, images=imgs, cameras=cams, depth=z, bgr=bgr))
        for key in [k for k in cache if last[k] == i]:
            del cache[key]
    return ring, problems
