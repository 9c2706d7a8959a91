"""Shared helpers of the GPU parity tests."""
import numpy as np

from crystalgraphics_b200 import scenes


def small_instanced(instances=128, lights=300, seed=5):
    """The instanced configuration's shape at a size the oracle finishes in
    seconds."""
    return scenes.instanced_scene(width=96, height=64, spp=1, depth=4, instances=instances,
                                  lights=lights, seed=seed, mesh_scale=0.05, extent=10.0,
                                  camera_distance=35.0)


def ray_set(scene, n, seed=0):
    """A fixed seeded ray set: half from the camera through random pixels,
    half from random points inside the scene's bounds in random directions."""
    rng = np.random.default_rng(seed)
    P = scene.vertices["position"]
    inst = scene.instances
    lo = np.full(3, np.inf)
    hi = np.full(3, -np.inf)
    for k in range(len(inst)):
        m = inst[k]["world_from_local"].reshape(3, 4).astype(np.float64)
        mesh = scene.meshes[inst[k]["mesh"]]
        v = P[mesh["vertex_offset"]:mesh["vertex_offset"] + mesh["vertex_count"]].astype(np.float64)
        w = v @ m[:, :3].T + m[:, 3]
        lo = np.minimum(lo, w.min(0))
        hi = np.maximum(hi, w.max(0))
    rays = np.zeros((n, 8), np.float32)
    half = n // 2
    cam = scene.camera
    o = np.array(cam.position[:], np.float64)
    d0 = np.array(cam.direction[:], np.float64)
    dx = np.cross(d0, [0, 0, 1.0])
    dx /= np.linalg.norm(dx)
    dy = np.cross(d0, dx)
    dy /= np.linalg.norm(dy)
    cx = rng.uniform(-1, 1, half) * cam.viewport[0]
    cy = rng.uniform(-1, 1, half) * cam.viewport[1]
    d = d0[None] + cx[:, None] * dx[None] + cy[:, None] * dy[None]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays[:half, :3] = o
    rays[:half, 4:7] = d
    m = n - half
    rays[half:, :3] = rng.uniform(lo, hi, (m, 3))
    dd = rng.normal(size=(m, 3))
    dd /= np.linalg.norm(dd, axis=1, keepdims=True)
    rays[half:, 4:7] = dd
    return rays


def camera_rays(camera, W, H):
    """cameraRay (compute.wesl:64-79) for every pixel, in float32."""
    f = np.float32
    d = np.array(camera.direction[:], f)
    dx = np.cross(d, np.array([0, 0, 1], f)).astype(f)
    dx = (dx / np.sqrt(np.sum(dx * dx, dtype=f))).astype(f) * f(camera.viewport[0])
    dy = np.cross(d, dx).astype(f)
    dy = (dy / np.sqrt(np.sum(dy * dy, dtype=f))).astype(f) * f(camera.viewport[1])
    px, py = np.meshgrid(np.arange(W, dtype=f), np.arange(H, dtype=f))
    cx = (px / f(W) * f(2) - f(1))[..., None]
    cy = (py / f(H) * f(2) - f(1))[..., None]
    r = (d + cx * dx + cy * dy).astype(f)
    r = r / np.sqrt(np.sum(r * r, axis=-1, keepdims=True, dtype=f))
    rays = np.zeros((H * W, 8), f)
    rays[:, :3] = np.array(camera.position[:], f)
    rays[:, 4:7] = r.reshape(-1, 3)
    return rays


def primary_tie_mask(oracle_scene, camera, W, H, ulps=4):
    """Pixels whose camera ray meets two surfaces at the same distance (within
    `ulps`): the closest hit there depends on traversal order (the reference
    keeps the first one it finds), so such pixels are excluded from image
    comparisons and counted, like ties in the hit-id comparison."""
    hits, t2 = oracle_scene.trace_closest(camera_rays(camera, W, H))
    t = hits["t"]
    tie = (hits["instance"] >= 0) & (np.abs(t2 - t) <= ulps * np.spacing(t))
    return tie.reshape(H, W)


def pooled(img, k):
    h, w, c = img.shape
    return img[:h - h % k, :w - w % k].reshape(h // k, k, w // k, k, c).mean(axis=(1, 3))


def pooled_masked(img, keep, k):
    """k x k block means over the pixels where `keep` is set."""
    h, w, c = img.shape
    m = keep[:h - h % k, :w - w % k].reshape(h // k, k, w // k, k, 1).astype(np.float64)
    x = img[:h - h % k, :w - w % k].reshape(h // k, k, w // k, k, c) * m
    return x.sum(axis=(1, 3)) / np.maximum(m.sum(axis=(1, 3)), 1)


def keyed_compare(gpu, ora, keep, tol=1e-3):
    """GPU film vs oracle film rendered from the same keyed sample streams, on
    X, Y and Z.  Each channel is scaled by the oracle's mean magnitude of that
    channel over the kept pixels.  Returns (fraction of kept pixel-channels
    within `tol`, the largest relative difference of a channel's mean, the
    scaled differences beyond `tol`)."""
    g = gpu[keep].reshape(-1, 3).astype(np.float64)
    o = ora[keep].reshape(-1, 3).astype(np.float64)
    scale = np.maximum(np.abs(o).mean(0), 1e-6)
    diff = (g - o) / scale
    close = float((np.abs(diff) <= tol).mean())
    rel_mean = float(np.max(np.abs(g.mean(0) - o.mean(0)) / scale))
    far = diff[np.abs(diff) > tol]
    return close, rel_mean, far
