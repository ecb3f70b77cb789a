"""PerspectiveCamera of the scene API (src/liar/cameras/perspective_camera.cpp)."""
from __future__ import annotations

import math

import numpy as np


def _unit(v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


class PerspectiveCamera:
    """Pinhole / thin-lens camera with the reference's parametrisation: width 0.036 m, aspect
    ratio 4/3, 90 degree field of view, sky (0, 0, 1), looking at (0, 1, 0) by default."""

    def __init__(self):
        self.position = (0.0, 0.0, 0.0)
        self._sky = np.array([0.0, 0.0, 1.0])
        self._width = 0.036
        self._height = self._width / (4.0 / 3.0)
        self._focal = (self._width / 2) / math.tan(math.pi / 4)
        self.nearLimit = 0.0
        self.farLimit = 3.4028234663852886e38
        self.lensRadius = 0.0
        self.focusDistance = 3.4028234663852886e38
        self.lookAt((0.0, 1.0, 0.0))

    # orientation
    @property
    def sky(self):
        return tuple(self._sky)

    @sky.setter
    def sky(self, v):
        self._sky = np.asarray(v, dtype=np.float64)

    @property
    def direction(self):
        return tuple(self._dir)

    @direction.setter
    def direction(self, d):
        # PerspectiveCamera::setDirection (perspective_camera.cpp:124-129)
        self._dir = _unit(d)
        self._right = _unit(np.cross(self._dir, self._sky))
        self._down = _unit(np.cross(self._dir, self._right))

    def lookAt(self, target):
        d = np.asarray(target, dtype=np.float64) - np.asarray(self.position, dtype=np.float64)
        self.direction = d
        self.focusDistance = float(np.linalg.norm(d))

    # film
    @property
    def width(self):
        return self._width

    @width.setter
    def width(self, w):
        self._width = float(w)

    @property
    def height(self):
        return self._height

    @height.setter
    def height(self, h):
        self._height = float(h)

    @property
    def aspectRatio(self):
        return self._width / self._height

    @aspectRatio.setter
    def aspectRatio(self, r):
        self._height = self._width / float(r)

    @property
    def focalLength(self):
        return self._focal

    @focalLength.setter
    def focalLength(self, f):
        self._focal = float(f)

    @property
    def fovAngle(self):
        return 2 * math.atan((self._width / 2) / self._focal)

    @fovAngle.setter
    def fovAngle(self, radians):
        self._focal = (self._width / 2) / math.tan(float(radians) / 2)

    def flatten(self):
        """The scaled basis the ray generator uses (PerspectiveCamera::initTransformation)."""
        return {
            "position": tuple(self.position),
            "direction": tuple(self._dir * self._focal),
            "right": tuple(self._right * self._width),
            "down": tuple(self._down * self._height),
            "direction_normal": tuple(self._dir),
            "right_normal": tuple(self._right),
            "down_normal": tuple(self._down),
            "lens_radius": float(self.lensRadius),
            "focus_distance": float(self.focusDistance) if self.lensRadius > 0 else 3.4028234663852886e38,
            "near_limit": float(self.nearLimit),
            "far_limit": float(self.farLimit),
        }
