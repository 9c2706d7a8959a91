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


def pooled(img, k):
    h, w, c = img.shape
    return img[:h - h % k, :w - w % k].reshape(h // k, k, w // k, k, c).mean(axis=(1, 3))
