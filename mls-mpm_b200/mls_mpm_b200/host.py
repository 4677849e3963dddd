"""Host-side logic of FluidGPU / DiffuseGPU that the reference runs in
JavaScript before each upload: uniform packing, the moving-wall packing with
velocity derivation, the hand dispatch box, and lineBoxIntersect.

JavaScript numbers are IEEE doubles and Float32Array stores round to nearest;
Python floats are doubles and numpy float32 stores round the same way, so
the bytes produced here are the bytes the reference uploads.
"""
import math

import numpy as np

from .abi import MAX_WALLS, HandParams, Params, WallParams


def grid_dims(aspect_x, aspect_y, aspect_z, particle_radius):
    """FluidGPU constructor grid sizing (fluid-gpu.js:11-14)."""
    norm = 1 / (particle_radius * 4)
    return (math.ceil(aspect_x * norm), math.ceil(aspect_y * norm), math.ceil(aspect_z * norm))


def line_box_intersect(origin, d, bmin, bmax):
    """math.js:149-164: slab test for an infinite line; [tmin, tmax] or None."""
    tmin, tmax = -math.inf, math.inf
    for i in range(3):
        if abs(d[i]) < 1e-9:
            if origin[i] < bmin[i] or origin[i] > bmax[i]:
                return None
            continue
        t1 = (bmin[i] - origin[i]) / d[i]
        t2 = (bmax[i] - origin[i]) / d[i]
        if t1 > t2:
            t1, t2 = t2, t1
        tmin = max(tmin, t1)
        tmax = min(tmax, t2)
        if tmin > tmax:
            return None
    return [tmin, tmax]


def f32(x):
    return float(np.float32(x))


def pack_params(fl, dt):
    """_writeParamsBuffer (fluid-gpu.js:295-313)."""
    p = Params()
    p.grid_X, p.grid_Y, p.grid_Z = fl.grid_X_num, fl.grid_Y_num, fl.grid_Z_num
    p.particle_num = fl.active_particle_num
    p.dt = dt
    p.gravity = fl.GRAVITY
    p.rest_density = fl.REST_DENSITY
    p.stiffness = fl.STIFFNESS
    p.eos_power = fl.EOS_POWER
    p.viscosity = fl.VISCOSITY
    p.hard_min = fl.HARD_MIN
    p.hard_max_x, p.hard_max_y, p.hard_max_z = fl.HARD_MAX_X, fl.HARD_MAX_Y, fl.HARD_MAX_Z
    p.wall_min = fl.WALL_MIN
    p.wall_stiffness = fl.WALL_STIFFNESS
    p.lookahead_k = fl.LOOKAHEAD_K
    return p


class WallSlot:
    """One entry of FluidGPU.walls (fluid-gpu.js:64-69)."""

    def __init__(self):
        self.active = False
        self.min = np.zeros(3, np.float32)
        self.max = np.zeros(3, np.float32)
        self.theta = 0.0
        self.phi = 0.0


class WallPacker:
    """Moving-wall state and the _writeWallParams packing (fluid-gpu.js:52-103,
    337-413), including its dedup (uploads only when the bytes change)."""

    def __init__(self):
        self.walls = [WallSlot() for _ in range(MAX_WALLS)]
        self.prev_min = [np.zeros(3, np.float32) for _ in range(MAX_WALLS)]
        self.prev_theta = [0.0] * MAX_WALLS
        self.prev_phi = [0.0] * MAX_WALLS
        self.buf = np.zeros(4 + MAX_WALLS * 20, np.float32)
        self.prev_buf = np.full(4 + MAX_WALLS * 20, np.nan, np.float32)

    def set_wall(self, i, mn, mx):
        w = self.walls[i]
        if not w.active:
            self.prev_min[i][:] = np.asarray(mn[:3], np.float32)
            self.prev_theta[i] = w.theta
            self.prev_phi[i] = w.phi
        w.active = True
        w.min[:] = np.asarray(mn[:3], np.float32)
        w.max[:] = np.asarray(mx[:3], np.float32)

    def rotate_wall(self, i, d_theta, d_phi=0.0):
        if not self.walls[i].active:
            return
        self.walls[i].theta += d_theta
        self.walls[i].phi += d_phi

    def remove_wall(self, i):
        self.walls[i].active = False

    def pack(self, DT, grid, hard_min, hard_max):
        """Returns (WallParams, changed).  grid = (X, Y, Z), hard_max = (x, y, z)."""
        inv_dt = 1.0 / DT
        HM1 = hard_min + 1.0
        count = 0
        f = self.buf
        for i in range(MAX_WALLS):
            w = self.walls[i]
            prev = self.prev_min[i]
            vx = vy = vz = d_theta = d_phi = 0.0
            if w.active:
                vx = (float(w.min[0]) - float(prev[0])) * inv_dt
                vy = (float(w.min[1]) - float(prev[1])) * inv_dt
                vz = (float(w.min[2]) - float(prev[2])) * inv_dt
                d_theta = (w.theta - self.prev_theta[i]) * inv_dt
                d_phi = (w.phi - self.prev_phi[i]) * inv_dt
            prev[:] = w.min
            self.prev_theta[i] = w.theta
            self.prev_phi[i] = w.phi
            if not w.active:
                continue
            mn = [float(v) for v in w.min]
            mx = [float(v) for v in w.max]
            cx = (mn[0] + mx[0]) * 0.5
            cy = (mn[1] + mx[1]) * 0.5
            cz = (mn[2] + mx[2]) * 0.5
            cyw, syw = math.cos(w.theta), math.sin(w.theta)
            cp, sp = math.cos(w.phi), math.sin(w.phi)
            omx, omy, omz = d_phi * cyw, d_theta, -d_phi * syw
            lminx, lminy, lminz = mn[0] - cx, mn[1] - cy, mn[2] - cz
            lmaxx, lmaxy, lmaxz = mx[0] - cx, mx[1] - cy, mx[2] - cz
            pitch_aligned = abs(sp) < 0.05 and cp > 0.95
            if pitch_aligned:
                if mn[1] <= HM1:
                    lminy = -4.0 - cy
                if mx[1] >= hard_max[1] - 1.0:
                    lmaxy = grid[1] + 4.0 - cy
                if abs(syw) < 0.05 and cyw > 0.95:
                    if mn[0] <= HM1:
                        lminx = -4.0 - cx
                    if mn[2] <= HM1:
                        lminz = -4.0 - cz
                    if mx[0] >= hard_max[0] - 1.0:
                        lmaxx = grid[0] + 4.0 - cx
                    if mx[2] >= hard_max[2] - 1.0:
                        lmaxz = grid[2] + 4.0 - cz
            b = 4 + count * 20
            f[b:b + 20] = [cx, cy, cz, cyw, lminx, lminy, lminz, syw, lmaxx, lmaxy, lmaxz, cp,
                           vx, vy, vz, sp, omx, omy, omz, 0.0]
            count += 1
        f[0] = count
        # element-wise !== as in the reference: NaN never equals, -0 == 0
        same = bool(np.array_equal(f, self.prev_buf))
        wp = WallParams.from_buffer_copy(f.tobytes())
        if same:
            return wp, False
        self.prev_buf[:] = f
        return wp, True


def pack_hand(fl, pos, vel, radius, strength, active, eye, buf=None):
    """updateHand (fluid-gpu.js:479-527).  Returns (HandParams, dims) where dims
    is the dispatch box (_handBBoxDim*); the bbox fields keep their previous
    values when the box is not recomputed, as the reference's buffer does."""
    h = buf if buf is not None else HandParams()
    h.px, h.py, h.pz = pos[0], pos[1], pos[2]
    h.radius = radius
    h.vx, h.vy, h.vz = vel[0], vel[1], vel[2]
    h.is_on = 1 if active else 0
    h.strength = strength
    h.ex, h.ey, h.ez = eye[0], eye[1], eye[2]
    dims = [0, 0, 0]
    if active:
        dx, dy, dz = pos[0] - eye[0], pos[1] - eye[1], pos[2] - eye[2]
        dl = math.hypot(dx, dy, dz) or 1
        d = [dx / dl, dy / dl, dz / dl]
        R = radius
        seg = line_box_intersect(pos, d, [-R, -R, -R],
                                 [fl.grid_X_num + R, fl.grid_Y_num + R, fl.grid_Z_num + R])
        if seg:
            t0, t1 = seg
            p0 = [pos[i] + t0 * d[i] for i in range(3)]
            p1 = [pos[i] + t1 * d[i] for i in range(3)]
            gmax = (fl.grid_X_num, fl.grid_Y_num, fl.grid_Z_num)
            lo = [max(0, math.floor(min(p0[i], p1[i]) - R)) for i in range(3)]
            hi = [min(gmax[i] - 1, math.ceil(max(p0[i], p1[i]) + R)) for i in range(3)]
            h.bbox_min_x, h.bbox_min_y, h.bbox_min_z = lo
            h.bbox_max_x, h.bbox_max_y, h.bbox_max_z = hi
            dims = [max(0, hi[i] - lo[i] + 1) for i in range(3)]
    return h, dims
