"""Sedimenting droplets in Stokes flow: the reference's application driver
(fmm3d_mpi/droplets.cpp) over this evaluator.

Particles of radius eps in a fluid of unit viscosity each carry the force
(0, 0, -eps^2).  The right-hand side of the particle ODE (eval_rhs,
droplets.cpp:20-173) is k = f + 6 pi eps u, where u is the velocity that the
other particles' forces induce, summed by the FMM with the Stokes velocity
kernel (311, Stokeslet): the points are shifted and scaled into the root box
[0, 1)^3 (scale 1 / (max - min + 0.02), shift 0.01 - min over all
coordinates), evaluated there, and the result is multiplied by the scale (the
Stokeslet is homogeneous of degree -1).  Positions advance by the classical
fourth-order Runge-Kutta step (droplets.cpp:425-478).

The evaluator is set up again for every right-hand side (the points move).  One
handle serves every setup and the operator tables come from the process's
cache, where the reference creates a new FMM per right-hand side over its
shared operator manager.  Everything from the scaled positions to the new
positions stays on the GPU apart from the host copy of the positions for the
tree build.

Initial particles (droplets.cpp:203, 251-300): uniform in the unit ball by
rejection from the cube [-1, 1]^3, drawn from drand48 seeded with the rank (0
at one process), or two such balls one above the other (the second shifted by
4 in z).  Unless skipped, they are snapped to the centres of the 2^-30 cells of
the scaled frame, duplicates dropped and sorted in Morton order
(droplets.cpp:317-360, which calls DENDRO's removeDuplicates; its order is
restated as Morton order with z the most significant axis on every level).
"""
import math
import os
import time

import numpy as np
import torch

import fmmg

KERNEL = 311  # Stokes velocity kernel, mu = 1 (droplets.cpp:215-219)
_A48, _C48, _M48 = 0x5DEECE66D, 0xB, (1 << 48) - 1


class Drand48:
    """The POSIX drand48 generator: X <- (a X + c) mod 2^48 with
    a = 0x5DEECE66D, c = 0xB, srand48(s) setting X = s << 16 | 0x330E, and
    each draw X / 2^48.  Draws come in blocks: X_{n+j} = A_j X_n + C_j with
    the j-step multiplier and increment, evaluated in uint64 arithmetic, whose
    wrap-around modulo 2^64 keeps the result exact modulo 2^48."""

    BLOCK = 4096

    def __init__(self, seed=0):
        self.x = ((int(seed) & 0xFFFFFFFF) << 16) | 0x330E
        a = np.empty(self.BLOCK, dtype=np.uint64)
        c = np.empty(self.BLOCK, dtype=np.uint64)
        aj, cj = 1, 0
        for j in range(self.BLOCK):
            aj, cj = (aj * _A48) & _M48, (cj * _A48 + _C48) & _M48
            a[j], c[j] = aj, cj
        self._a, self._c = a, c

    def states(self, n):
        """The next n generator states (uint64), advancing the generator."""
        out = np.empty(n, dtype=np.uint64)
        done = 0
        while done < n:
            m = min(self.BLOCK, n - done)
            xs = (self._a[:m] * np.uint64(self.x) + self._c[:m]) & np.uint64(_M48)
            out[done:done + m] = xs
            self.x = int(xs[m - 1])
            done += m
        return out

    def draws(self, n):
        return self.states(n).astype(np.float64) * 2.0 ** -48


def _ball(gen, n):
    """n points uniform in the unit ball: triples 1 - 2 drand48() kept when
    inside (r^2 < 1), in the order the reference's loop draws them; the
    generator is left just after the last accepted triple."""
    parts, have = [], 0
    while have < n:
        need = n - have
        st = gen.states(3 * (2 * need + 64))
        t = 1.0 - 2.0 * (st.astype(np.float64) * 2.0 ** -48).reshape(-1, 3)
        inside = np.nonzero((t * t).sum(1) < 1.0)[0]
        if inside.size >= need:
            parts.append(t[inside[:need]])
            gen.x = int(st[3 * (inside[need - 1] + 1) - 1])
            have = n
        else:
            parts.append(t[inside])
            have += inside.size
    return np.concatenate(parts) if parts else np.empty((0, 3))


def initial_positions(n, distribution="ball", seed=0):
    """The reference's initial particles (droplets.cpp:203, 251-300)."""
    gen = Drand48(seed)
    if distribution == "ball":
        return _ball(gen, n)
    if distribution == "two_balls_vert":
        a = _ball(gen, n // 2)
        b = _ball(gen, n - n // 2)
        b[:, 2] += 4.0
        return np.concatenate([a, b])
    raise ValueError("distribution must be 'ball' or 'two_balls_vert'")


def box_map(x):
    """(scale, shift) taking the points into [0, 1)^3: x' = (x + shift) * scale
    (droplets.cpp:50-63)."""
    lo, hi = float(x.min()), float(x.max())
    return 1.0 / (hi - lo + 0.02), -lo + 0.01


def _morton(cells):
    key = np.zeros(cells.shape[0], dtype=np.uint64)
    for b in range(30):
        for d in range(3):  # x, y, z: z lands on the most significant bit of each level
            key |= ((cells[:, d] >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + d)
    return key


def snap_and_dedup(x):
    """Snap to the 2^-30 cell centres of the scaled frame, drop duplicates and
    sort in Morton order (droplets.cpp:317-360)."""
    scale, shift = box_map(x)
    u = (np.asarray(x, dtype=np.float64) + shift) * scale
    cells = np.ldexp(u, 30).astype(np.uint64)  # unsigned(ldexp(p, 30)): truncation
    key = _morton(cells)
    _, first = np.unique(key, return_index=True)  # sorted by key, one per cell
    c = cells[first].astype(np.float64)
    return np.ldexp(c + 0.5, -30) / scale - shift


def particle_size(n, volume_ratio):
    """eps from the volume fraction (droplets.cpp:383-400)."""
    return math.exp(math.log(volume_ratio / n) / 3.0)


def rk4_step(x, rhs, h):
    """x + h/6 (k1 + 2 k2 + 2 k3 + k4) (droplets.cpp:425-462)."""
    k1 = rhs(x)
    k2 = rhs(x + (h / 2) * k1)
    k3 = rhs(x + (h / 2) * k2)
    k4 = rhs(x + h * k3)
    return x + (h / 6) * k1 + (h / 3) * k2 + (h / 3) * k3 + (h / 6) * k4


class FmmVelocity:
    """Stokeslet velocities of point forces through one fmmg handle on a GPU:
    __call__(scaled positions (n, 3) CUDA float64, forces (n*3,)) -> (n, 3)."""

    def __init__(self, np_=6, pts_max=64, precision=fmmg.PREC_FP64, device=0):
        self.f = fmmg.FMM3d(KERNEL, np_=np_, pts_max=pts_max, coefs=(1.0, 0.25), device=device)
        self.precision = precision
        self.device = torch.device("cuda", device)
        self.setup_s = self.evaluate_s = 0.0  # wall time spent in each, summed over calls

    def __call__(self, xs, den):
        t0 = time.perf_counter()
        self.f.setup(xs.detach().cpu().numpy())
        t1 = time.perf_counter()
        out = torch.empty(den.numel(), dtype=torch.float64, device=self.device)
        self.f.evaluate_device(den, out, 1, self.precision)
        self.f.sync()
        self.setup_s += t1 - t0
        self.evaluate_s += time.perf_counter() - t1
        return out.view(-1, 3)


class Droplets:
    """State and time stepping of the droplets problem.  `velocity(xs, den)`
    returns the FMM velocities at the scaled positions xs (default: FmmVelocity
    on cuda:0); positions live in a float64 tensor on the device velocity
    works on."""

    def __init__(self, x, eps, h, velocity=None, device=None):
        self.velocity = velocity if velocity is not None else FmmVelocity()
        dev = device if device is not None else getattr(self.velocity, "device", torch.device("cpu"))
        self.x = torch.as_tensor(np.asarray(x, dtype=np.float64), device=dev).contiguous()
        self.eps, self.h = float(eps), float(h)
        self.den = torch.zeros_like(self.x)
        self.den[:, 2] = -self.eps * self.eps  # droplets.cpp:99-106
        self.den_flat = self.den.view(-1)
        self.evaluations = 0

    def rhs(self, x):
        """k = f + 6 pi eps u(x) (droplets.cpp:20-173)."""
        scale, shift = box_map(x)
        xs = ((x + shift) * scale).contiguous()
        u = self.velocity(xs, self.den_flat)
        self.evaluations += 1
        return self.den + (6.0 * math.pi * self.eps * scale) * u

    def step(self):
        self.x = rk4_step(self.x, self.rhs, self.h)
        return self.x

    def run(self, num_iter, write_fraction=0, out_dir=None):
        """num_iter RK4 steps; with out_dir, the positions are written before
        the first step and after every write_fraction-th one as
        coord<i>.txt, one 'x y z' line per particle."""
        if out_dir:
            os.makedirs(out_dir, exist_ok=True)
            self.write(os.path.join(out_dir, "coord0.txt"))
        for i in range(1, num_iter + 1):
            self.step()
            if out_dir and write_fraction and i % write_fraction == 0:
                self.write(os.path.join(out_dir, "coord%d.txt" % i))
        return self.x

    def write(self, path):
        np.savetxt(path, self.x.detach().cpu().numpy(), fmt="%.17g")


def main(argv=None):
    """Command line of the reference driver: -numsrc, -distribution,
    -time_step, -particle_size or -volume_ratio, -num_iter, -write_fraction,
    -skip_initial_sort, -preserve_order, -isogranular (droplets.cpp:176-410)."""
    import argparse
    p = argparse.ArgumentParser(description=main.__doc__)
    p.add_argument("--numsrc", type=int, required=True)
    p.add_argument("--distribution", choices=("ball", "two_balls_vert"), required=True)
    p.add_argument("--time_step", type=float, required=True)
    g = p.add_mutually_exclusive_group(required=True)
    g.add_argument("--particle_size", type=float)
    g.add_argument("--volume_ratio", type=float)
    p.add_argument("--num_iter", type=int, required=True)
    p.add_argument("--write_fraction", type=int, required=True)
    p.add_argument("--skip_initial_sort", action="store_true")
    # at one process these change nothing: the evaluator returns values in the
    # caller's order (-preserve_order, droplets.cpp:407) and -numsrc is the
    # process's own count either way (-isogranular, :221-247)
    p.add_argument("--preserve_order", action="store_true")
    p.add_argument("--isogranular", action="store_true")
    p.add_argument("--np", type=int, default=6)
    p.add_argument("--pts_max", type=int, default=64)
    p.add_argument("--mixed", action="store_true", help="evaluate in the mixed-precision form")
    p.add_argument("--out", default=None, help="folder for the coord<i>.txt files (none: not written)")
    a = p.parse_args(argv)
    x = initial_positions(a.numsrc, a.distribution)
    if not a.skip_initial_sort:
        x = snap_and_dedup(x)
    eps = a.particle_size if a.particle_size is not None else particle_size(x.shape[0], a.volume_ratio)
    vel = FmmVelocity(a.np, a.pts_max, fmmg.PREC_MIXED if a.mixed else fmmg.PREC_FP64)
    d = Droplets(x, eps, a.time_step, vel)
    print("particles %d, particle size %g, time step %g, iterations %d" % (x.shape[0], eps, a.time_step, a.num_iter))
    t0 = time.perf_counter()
    d.run(a.num_iter, a.write_fraction, a.out)
    wall = time.perf_counter() - t0
    print("%d steps (%d right-hand sides) in %.3f s: setup %.3f s, evaluate %.3f s, the rest %.3f s"
          % (a.num_iter, d.evaluations, wall, vel.setup_s, vel.evaluate_s, wall - vel.setup_s - vel.evaluate_s))


if __name__ == "__main__":
    main()
