"""Deterministic scenario generators.

Two families:

* Ports of the reference's FROZEN fixtures (crates/pf_core/src/sim.rs): the
  xorshift ``Gauss`` source, ``landmark_box``, ``circle_scenario`` and
  ``room_grid``.  Their draw order defines the reference's test scenarios,
  so they are restated operation for operation.
* Generators for the benchmark workloads: a helix trajectory with point
  landmarks (plain and at-scale PF cycles, optionally with uniform outlier
  observations) and a walled 10 x 10 m room with random box obstacles for
  global localization.  All draws come from one numpy PCG64 stream per seed.

Quaternions are (w, x, y, z) Hamilton, as in the library.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MASK64 = (1 << 64) - 1


# ---------------------------------------------------------------- quaternions

def qmul(a, b):
    aw, ax, ay, az = a
    bw, bx, by, bz = b
    return np.array([aw * bw - ax * bx - ay * by - az * bz,
                     aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw])


def qconj(q):
    return np.array([q[0], -q[1], -q[2], -q[3]])


def qrot(q, v):
    """v' = v + 2w(u x v) + 2u x (u x v)."""
    u = np.asarray(q[1:], dtype=float)
    t = 2.0 * np.cross(u, v)
    return np.asarray(v, dtype=float) + q[0] * t + np.cross(u, t)


def qinvrot(q, v):
    return qrot(qconj(q), v)


def qinvrot_rows(q, v):
    """qinvrot applied to every row of v (k, 3)."""
    qc = qconj(q)
    u = np.asarray(qc[1:], dtype=float)
    t = 2.0 * np.cross(u[None, :], v)
    return v + qc[0] * t + np.cross(u[None, :], t)


def q_axis_angle(axis, angle):
    axis = np.asarray(axis, dtype=float)
    n = np.linalg.norm(axis)
    if not angle > 1e-12 or not n > 1e-12:
        return np.array([1.0, 0.0, 0.0, 0.0])
    s = math.sin(0.5 * angle) / n
    return np.array([math.cos(0.5 * angle), axis[0] * s, axis[1] * s, axis[2] * s])


def q_yaw(yaw):
    return np.array([math.cos(0.5 * yaw), 0.0, 0.0, math.sin(0.5 * yaw)])


# --------------------------------------------------------------- containers

@dataclass
class Step:
    odom_t: np.ndarray           # body-frame translation (3,)
    odom_q: np.ndarray           # rotation (w,x,y,z)
    obs: np.ndarray              # (k, 6): id, mode, dx, dy, dz, range
    truth_p: np.ndarray          # true position after the motion
    truth_q: np.ndarray


@dataclass
class Scenario:
    landmarks: np.ndarray        # (L, 3), dense by id
    prior_p: np.ndarray
    prior_q: np.ndarray
    steps: list = field(default_factory=list)
    trans_noise: tuple = (0.05, 0.05, 0.05)
    rot_noise: tuple = (0.02, 0.02, 0.03)

    def landmark_dict(self):
        return {i: self.landmarks[i] for i in range(len(self.landmarks))}


# ------------------------------------------------------ frozen sim.rs ports

class Gauss:
    """xorshift64 noise source of crates/pf_core/src/sim.rs:14-42."""

    def __init__(self, seed: int):
        self.s = seed & MASK64

    def _step(self):
        s = self.s
        s ^= (s << 13) & MASK64
        s ^= s >> 7
        s ^= (s << 17) & MASK64
        self.s = s
        return s

    def next_box(self) -> float:
        return (self._step() % 8000) / 1000.0 + 1.0

    def next01(self) -> float:
        return (self._step() % 10000) / 10000.0

    def normal(self) -> float:
        return (self.next01() + self.next01() - 1.0) * 1.732


def landmark_box(n: int, seed: int) -> np.ndarray:
    """sim.rs:44-52: n landmarks in an ~8 x 8 x 2.4 m box."""
    g = Gauss(seed)
    out = np.zeros((n, 3))
    for i in range(n):
        x = g.next_box()
        y = g.next_box()
        z = g.next_box() * 0.3
        out[i] = (x, y, z)
    return out


def circle_scenario(steps_n: int, seed: int) -> Scenario:
    """sim.rs:69-121: circular climb, Cartesian observations within 5 m."""
    lm = landmark_box(12, 99)
    prior_p = np.array([5.0, 5.0, 0.5])
    prior_q = np.array([1.0, 0.0, 0.0, 0.0])
    g = Gauss(seed)
    dt = 0.1
    tp, tq = prior_p.copy(), prior_q.copy()
    sc = Scenario(lm, prior_p, prior_q)
    for t in range(steps_n):
        vel = np.array([-0.4 * math.sin(0.2 * t * dt), 0.4 * math.cos(0.2 * t * dt), 0.02])
        yaw = math.atan2(vel[1], vel[0])
        att = q_yaw(yaw)  # UnitQuaternion::from_axis_angle(z, yaw)
        new_p = tp + vel * dt
        odo_t = qinvrot(tq, new_p - tp)
        odo_q = qmul(qconj(tq), att)
        odo_t = odo_t + np.array([g.normal() * 0.05, g.normal() * 0.05, g.normal() * 0.05])
        tp, tq = new_p, att
        obs = []
        for i in range(len(lm)):
            body = qinvrot(tq, lm[i] - tp)
            d = float(np.linalg.norm(body))
            if d > 5.0:
                continue
            noisy = body * (1.0 + g.normal() * 0.05 / max(d, 0.1))
            obs.append((i, 0, noisy[0], noisy[1], noisy[2], 0.0))
        sc.steps.append(Step(odo_t, odo_q, np.array(obs, dtype=float).reshape(-1, 6),
                             tp.copy(), tq.copy()))
    return sc


def room_grid() -> np.ndarray:
    """sim.rs:123-151: 200 x 200 room at 0.05 m, walls + pillar at (4, 5)."""
    w = h = 200
    cells = np.zeros((h, w), dtype=np.uint8)
    cells[0, :] = 1
    cells[h - 1, :] = 1
    cells[:, 0] = 1
    cells[:, w - 1] = 1
    x0, x1 = int((4.0 - 0.25) / 0.05), int((4.0 + 0.25) / 0.05)
    y0, y1 = int((5.0 - 0.25) / 0.05), int((5.0 + 0.25) / 0.05)
    cells[y0:y1 + 1, x0:x1 + 1] = 1
    return cells


# ------------------------------------------------------- benchmark workloads

def helix_scenario(cycles: int, n_landmarks: int, box: tuple, n_obs: int | None = None,
                   outlier_frac: float = 0.0, seed: int = 1, obs_sigma: float = 0.05,
                   odo_sigma_t: float = 0.02, odo_sigma_r: float = 0.01,
                   radius: float = 5.0, arc: float = 0.1, climb: float = 0.005,
                   phase: float = 0.0) -> Scenario:
    """Helix trajectory (radius 5 m, 0.1 m of arc and arc/radius rad of yaw per
    step, 0.005 m climb per step) through a landmark box centred on the helix
    axis.  Each cycle observes either every landmark (n_obs None) or n_obs
    observations with ids uniform over the landmarks (repeats allowed), a
    fraction of which are outliers: a random id whose vector points at a
    uniform point of the box.  Odometry is the true body-frame delta plus
    N(0, odo_sigma_t) per axis and an axis-angle rotation of N(0,
    odo_sigma_r) per axis; Cartesian observations carry N(0, obs_sigma) per
    axis.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    bx, by, bz = box
    centre = np.array([0.0, 0.0, bz / 2.0])
    lm = rng.uniform([-bx / 2, -by / 2, 0.0], [bx / 2, by / 2, bz], size=(n_landmarks, 3))
    dyaw = arc / radius

    def pose(k):
        ang = phase + k * dyaw
        p = centre + np.array([radius * math.cos(ang), radius * math.sin(ang),
                               -bz / 4.0 + climb * k])
        return p, q_yaw(ang + math.pi / 2.0)

    tp, tq = pose(0)
    sc = Scenario(lm, tp.copy(), tq.copy(), trans_noise=(odo_sigma_t,) * 3,
                  rot_noise=(odo_sigma_r,) * 3)
    for k in range(1, cycles + 1):
        np_, nq = pose(k)
        odo_t = qinvrot(tq, np_ - tp) + rng.normal(0.0, odo_sigma_t, 3)
        dq = qmul(qconj(tq), nq)
        w = rng.normal(0.0, odo_sigma_r, 3)
        odo_q = qmul(dq, q_axis_angle(w, float(np.linalg.norm(w))))
        tp, tq = np_, nq
        if n_obs is None:
            ids = np.arange(n_landmarks)
            n_out = 0
        else:
            n_out = int(round(outlier_frac * n_obs))
            ids = rng.integers(0, n_landmarks, size=n_obs)
        rows = np.zeros((len(ids), 6))
        rows[:, 0] = ids
        n_in = len(ids) - n_out
        world = np.empty((len(ids), 3))
        world[:n_in] = lm[ids[:n_in]] - tp
        if n_out:
            world[n_in:] = rng.uniform([-bx / 2, -by / 2, 0.0], [bx / 2, by / 2, bz],
                                       size=(n_out, 3)) - tp
        rows[:, 2:5] = qinvrot_rows(tq, world)
        rows[:n_in, 2:5] += rng.normal(0.0, obs_sigma, size=(n_in, 3))
        if n_out:
            perm = rng.permutation(len(ids))
            rows = rows[perm]
        sc.steps.append(Step(odo_t, odo_q, rows, tp.copy(), tq.copy()))
    return sc


def as_range_bearing(sc: Scenario) -> Scenario:
    """The same scenario with every observation in range-bearing form (mode
    1): range |v| and the unit direction -v/|v| of the body-frame vector v
    (the measurement model compares the direction with -pred / |pred|,
    src/cuda/pf_kernels.cu:253-268), the Cartesian noise carried over."""
    out = Scenario(sc.landmarks, sc.prior_p, sc.prior_q, trans_noise=sc.trans_noise,
                   rot_noise=sc.rot_noise)
    for st in sc.steps:
        rows = st.obs.copy()
        v = rows[:, 2:5]
        r = np.linalg.norm(v, axis=1)
        rows[:, 1] = 1
        rows[:, 5] = r
        rows[:, 2:5] = -v / np.maximum(r, 1e-9)[:, None]
        out.steps.append(Step(st.odom_t, st.odom_q, rows, st.truth_p, st.truth_q))
    return out


def tracking_config(cycles=100, seed=7) -> Scenario:
    """Plain PF tracking workload: 12 landmarks in a 20 x 20 x 5 m box, every
    landmark observed each cycle, 3-sigma gate, 0.02 m / 0.01 rad odometry."""
    return helix_scenario(cycles, 12, (20.0, 20.0, 5.0), None, 0.0, seed)


def scale_config(cycles=1000, seed=11) -> Scenario:
    """At-scale PF workload: 64 landmarks in a 50 x 50 x 10 m box, 256
    observations per cycle of which 10 % are uniform outliers."""
    return helix_scenario(cycles, 64, (50.0, 50.0, 10.0), 256, 0.10, seed)


def rooms_grid(seed: int, n_boxes: int = 30, size_m: float = 10.0,
               res: float = 0.05) -> np.ndarray:
    """Walled rectangular room (one-cell walls) with n_boxes axis-aligned box
    obstacles of side U[0.2, 1.0] m at uniform centres; boxes are redrawn
    while they would leave less than half of the interior free."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = int(round(size_m / res))
    cells = np.zeros((n, n), dtype=np.uint8)
    cells[0, :] = cells[-1, :] = 1
    cells[:, 0] = cells[:, -1] = 1
    placed = 0
    while placed < n_boxes:
        sx, sy = rng.uniform(0.2, 1.0, 2)
        cx, cy = rng.uniform(0.0, size_m, 2)
        x0 = max(1, int((cx - sx / 2) / res))
        x1 = min(n - 2, int((cx + sx / 2) / res))
        y0 = max(1, int((cy - sy / 2) / res))
        y1 = min(n - 2, int((cy + sy / 2) / res))
        if x1 < x0 or y1 < y0:
            continue
        trial = cells.copy()
        trial[y0:y1 + 1, x0:x1 + 1] = 1
        if (trial[1:-1, 1:-1] == 0).mean() < 0.5:
            continue
        cells = trial
        placed += 1
    return cells


def free_pose(cells: np.ndarray, rng: np.random.Generator, res=0.05, origin=(0.0, 0.0),
              margin_cells: int = 2):
    """Uniform free cell (at least margin_cells away from any obstacle) +
    uniform in-cell offset, yaw uniform in [0, 2 pi)."""
    occ = cells != 0
    pad = np.pad(occ, margin_cells, constant_values=True)
    near = np.zeros_like(occ)
    h, w = occ.shape
    for dy in range(-margin_cells, margin_cells + 1):
        for dx in range(-margin_cells, margin_cells + 1):
            near |= pad[margin_cells + dy:margin_cells + dy + h,
                        margin_cells + dx:margin_cells + dx + w]
    ys, xs = np.nonzero(~near)
    k = rng.integers(0, len(xs))
    x = origin[0] + (xs[k] + rng.uniform()) * res
    y = origin[1] + (ys[k] + rng.uniform()) * res
    return float(x), float(y), float(rng.uniform(0.0, 2 * math.pi))


def batched_config(n_filters: int = 512, cycles: int = 200, seed: int = 23,
                   n_min: int = 1000, n_max: int = 200_000):
    """Batched PF workload: n_filters independent filters with N drawn
    log-uniform in [n_min, n_max], each with its own 8-64 landmarks in a
    20 x 20 x 5 m box and its own helix (random phase), and 4-64 observations
    per cycle.  Returns (sizes, scenarios, nobs[f][cycle])."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = np.exp(rng.uniform(math.log(n_min), math.log(n_max), n_filters)).astype(int)
    scen, counts = [], []
    for f in range(n_filters):
        n_lm = int(rng.integers(8, 65))
        sc = helix_scenario(cycles, n_lm, (20.0, 20.0, 5.0), 64, 0.0,
                            int(rng.integers(1, 1 << 31)),
                            phase=float(rng.uniform(0.0, 2 * math.pi)))
        c = rng.integers(4, 65, size=cycles)
        for k, st in enumerate(sc.steps):
            st.obs = st.obs[: int(c[k])]
        scen.append(sc)
        counts.append(c)
    return sizes, scen, np.array(counts)
