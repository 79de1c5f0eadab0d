"""The viewer's camera and matrices (src/render.js:5-100, 202-258): an orbit camera
around a target, perspective(FOVY = 45 deg, aspect, 0.05, 100), lookAt, the 4x4
inverse, and the invView the renderer builds from the camera basis. Column-major
lists of 16, computed in double as the JS does; the render passes take them as
float32.

    cam = Camera(); cam.frame(box)
    m = frame_matrices(cam, width, height)   # view, proj, inv_view_proj, inv_view, eye
"""
import math

FOVY = 45 * math.pi / 180


def _sub(a, b):
    return [a[0] - b[0], a[1] - b[1], a[2] - b[2]]


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _norm(a):
    l = math.hypot(*a) or 1.0
    return [a[0] / l, a[1] / l, a[2] / l]


def perspective(fovy, aspect, near, far):
    """src/render.js:5-12 (OpenGL-style depth range)."""
    f = 1 / math.tan(fovy / 2)
    nf = 1 / (near - far)
    return [f / aspect, 0, 0, 0, 0, f, 0, 0, 0, 0, (far + near) * nf, -1, 0, 0, 2 * far * near * nf, 0]


def look_at(eye, target, up):
    """src/render.js:13-21."""
    z = _norm(_sub(eye, target))
    x = _norm(_cross(up, z))
    y = _cross(z, x)
    return [x[0], y[0], z[0], 0, x[1], y[1], z[1], 0, x[2], y[2], z[2], 0,
            -_dot(x, eye), -_dot(y, eye), -_dot(z, eye), 1]


def mul(a, b):
    """src/render.js:27-33: column-major a * b."""
    o = [0.0] * 16
    for c in range(4):
        for r in range(4):
            for k in range(4):
                o[c * 4 + r] += a[k * 4 + r] * b[c * 4 + k]
    return o


def inverse(m):
    """src/render.js:35-64 (cofactor expansion; a singular matrix gives zeros)."""
    a00, a01, a02, a03, a10, a11, a12, a13, a20, a21, a22, a23, a30, a31, a32, a33 = m
    b00 = a00 * a11 - a01 * a10
    b01 = a00 * a12 - a02 * a10
    b02 = a00 * a13 - a03 * a10
    b03 = a01 * a12 - a02 * a11
    b04 = a01 * a13 - a03 * a11
    b05 = a02 * a13 - a03 * a12
    b06 = a20 * a31 - a21 * a30
    b07 = a20 * a32 - a22 * a30
    b08 = a20 * a33 - a23 * a30
    b09 = a21 * a32 - a22 * a31
    b10 = a21 * a33 - a23 * a31
    b11 = a22 * a33 - a23 * a32
    det = b00 * b11 - b01 * b10 + b02 * b09 + b03 * b08 - b04 * b07 + b05 * b06
    d = 1 / det if det else 0
    return [(a11 * b11 - a12 * b10 + a13 * b09) * d, (a02 * b10 - a01 * b11 - a03 * b09) * d,
            (a31 * b05 - a32 * b04 + a33 * b03) * d, (a22 * b04 - a21 * b05 - a23 * b03) * d,
            (a12 * b08 - a10 * b11 - a13 * b07) * d, (a00 * b11 - a02 * b08 + a03 * b07) * d,
            (a32 * b02 - a30 * b05 - a33 * b01) * d, (a20 * b05 - a22 * b02 + a23 * b01) * d,
            (a10 * b10 - a11 * b08 + a13 * b06) * d, (a01 * b08 - a00 * b10 - a03 * b06) * d,
            (a30 * b04 - a31 * b02 + a33 * b00) * d, (a21 * b02 - a20 * b04 - a23 * b00) * d,
            (a11 * b07 - a10 * b09 - a12 * b06) * d, (a00 * b09 - a01 * b07 + a02 * b06) * d,
            (a31 * b01 - a30 * b03 - a32 * b00) * d, (a20 * b03 - a21 * b01 + a22 * b00) * d]


class Camera:
    """src/render.js:68-98: azimuth / elevation orbit at `dist` around `target`."""

    def __init__(self):
        self.az, self.el, self.dist = -0.5, 0.35, 2.2
        self.target = [0.5, 0.4, 0.3]

    def frame(self, box):
        self.target = [box[0] / 2, box[1] / 2, box[2] / 2]
        self.dist = 1.8 * max(box[0], box[1], box[2])
        return self

    def eye_dir(self):
        ce, se = math.cos(self.el), math.sin(self.el)
        return [ce * math.sin(self.az), se, ce * math.cos(self.az)]

    def eye(self):
        d = self.eye_dir()
        return [self.target[k] + self.dist * d[k] for k in range(3)]


def frame_matrices(cam, width, height):
    """The matrices src/render.js:203-258 hands to FluidSSFR.render."""
    eye = cam.eye()
    proj = perspective(FOVY, width / max(1, height), 0.05, 100)
    view = look_at(eye, cam.target, [0, 1, 0])
    vp = mul(proj, view)
    fwd = _norm(_sub(cam.target, eye))
    right = _norm(_cross(fwd, [0, 1, 0]))
    up = _norm(_cross(right, fwd))
    inv_view = [right[0], right[1], right[2], 0, up[0], up[1], up[2], 0,
                -fwd[0], -fwd[1], -fwd[2], 0, eye[0], eye[1], eye[2], 1]
    return {"view": view, "proj": proj, "inv_view_proj": inverse(vp), "inv_view": inv_view, "eye": eye,
            "width": int(width), "height": int(height)}
