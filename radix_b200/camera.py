"""Cameras as the C ABI takes them: float64 4x4 matrices, column-major.

perspective() and look_at() build what a three.js PerspectiveCamera holds
(vertical field of view, camera looking down -z with +y up, projection in the
WebGPU clip convention by default: NDC z in [0, 1]). They are the standard
constructions; the ABI takes any view and projection matrices.
"""
import math

import numpy as np


def perspective(fov_deg, aspect, near, far, webgpu=True):
    """Projection of a symmetric frustum, column-major float64[16]."""
    top = near * math.tan(math.radians(fov_deg) * 0.5)
    bottom = -top
    right = top * aspect
    left = -right
    m = np.zeros((4, 4))
    m[0, 0] = 2 * near / (right - left)
    m[1, 1] = 2 * near / (top - bottom)
    m[0, 2] = (right + left) / (right - left)
    m[1, 2] = (top + bottom) / (top - bottom)
    if webgpu:  # z_ndc in [0, 1]
        m[2, 2] = -far / (far - near)
        m[2, 3] = -far * near / (far - near)
    else:  # z_ndc in [-1, 1]
        m[2, 2] = -(far + near) / (far - near)
        m[2, 3] = -2 * far * near / (far - near)
    m[3, 2] = -1.0
    return m.T.reshape(16).copy()  # column-major


def look_at_world(eye, target, up=(0.0, 1.0, 0.0)):
    """Camera -> world (matrixWorld) of a camera at `eye` whose -z faces `target`."""
    eye = np.asarray(eye, dtype=np.float64)
    z = eye - np.asarray(target, dtype=np.float64)
    z /= np.linalg.norm(z)
    x = np.cross(np.asarray(up, dtype=np.float64), z)
    if np.linalg.norm(x) < 1e-12:  # looking along up: nudge as three.js does
        z = z + np.array([1e-4, 0.0, 0.0])
        z /= np.linalg.norm(z)
        x = np.cross(np.asarray(up, dtype=np.float64), z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    m = np.eye(4)
    m[:3, 0] = x
    m[:3, 1] = y
    m[:3, 2] = z
    m[:3, 3] = eye
    return m.T.reshape(16).copy()


def invert(m16):
    """Inverse of a column-major 4x4."""
    m = np.asarray(m16, dtype=np.float64).reshape(4, 4).T
    return np.linalg.inv(m).T.reshape(16).copy()


def look_at(eye, target, up=(0.0, 1.0, 0.0)):
    """World -> camera (matrixWorldInverse), column-major float64[16]."""
    return invert(look_at_world(eye, target, up))


def translation(x, y, z):
    m = np.eye(4)
    m[:3, 3] = (x, y, z)
    return m.T.reshape(16).copy()


def multiply(a16, b16):
    """a * b of column-major 4x4s."""
    a = np.asarray(a16, dtype=np.float64).reshape(4, 4).T
    b = np.asarray(b16, dtype=np.float64).reshape(4, 4).T
    return (a @ b).T.reshape(16).copy()


IDENTITY = np.eye(4).reshape(16).copy()


class Camera:
    """The camera of one render (SplatCamera.setViews): world -> head, 1 or 2
    eyes of (view, projection, ortho), one render size, the near-plane NDC z."""

    def __init__(self, head, eyes, width, height, ndc_z_min=0.0):
        if not 1 <= len(eyes) <= 2:
            raise ValueError(f"SplatCamera: 1 or 2 eyes, not {len(eyes)}")
        self.head = np.asarray(head, dtype=np.float64).reshape(16)
        self.eyes = [(np.asarray(v, dtype=np.float64).reshape(16), np.asarray(p, dtype=np.float64).reshape(16),
                      bool(o)) for v, p, o in eyes]
        self.width = float(width)
        self.height = float(height)
        self.ndc_z_min = float(ndc_z_min)

    @classmethod
    def mono(cls, eye, target, fov_deg, width, height, near=0.01, far=1000.0, up=(0.0, 1.0, 0.0)):
        """A plain PerspectiveCamera: one eye that is also the head."""
        view = look_at(eye, target, up)
        proj = perspective(fov_deg, width / height, near, far)
        return cls(view, [(view, proj, False)], width, height)

    @classmethod
    def stereo(cls, head_pos, target, fov_deg, width, height, baseline=0.064, near=0.01, far=1000.0,
               up=(0.0, 1.0, 0.0)):
        """Two eyes at -/+ baseline/2 along the head's x, the head at their midpoint."""
        head_world = np.asarray(look_at_world(head_pos, target, up)).reshape(4, 4).T
        proj = perspective(fov_deg, width / height, near, far)
        eyes = []
        for side in (-0.5, 0.5):
            eye_world = head_world @ np.asarray(translation(side * baseline, 0.0, 0.0)).reshape(4, 4).T
            eyes.append((invert(eye_world.T.reshape(16)), proj, False))
        return cls(invert(head_world.T.reshape(16)), eyes, width, height)

    def to_c(self, abi):
        c = abi.rdx_camera()
        c.head[:] = list(self.head)
        c.eyes = len(self.eyes)
        for v, (view, proj, ortho) in enumerate(self.eyes):
            c.eye[v].view[:] = list(view)
            c.eye[v].projection[:] = list(proj)
            c.eye[v].ortho = 1 if ortho else 0
        c.width = self.width
        c.height = self.height
        c.ndc_z_min = self.ndc_z_min
        return c
