"""FP64 host reference for the gradient of the electrostatic step (test
infrastructure: the checker of aw_grad_es, never part of the product).

The reference has no adjoint. This module restates, in float64 and without the
fixed-point quantisation, the ES step the library runs, and its discrete
adjoint, so that the library's FP32 gradient has an FP64 reference, and the
FP64 reference itself is checked against central finite differences.

Forward (the reference's ES step, Simulation<Cfg>::step):
  rho   = CIC deposit of q_p = qm w_p / (dx dy)      include/pic/depositor.hpp:35-58
  E     = spectral Poisson, E_k = -i k rho_k/(eps0 k^2), k = 0 and Nyquist zeroed
                                                      include/pic/solver_es.hpp:40-78
  u'    = Boris: half kick, rotation about B0, half kick   include/pic/pusher.hpp:47-80
  x'    = wrap(x + u' dt/dx)                          include/pic/pusher.hpp:126-127,
                                                      include/pic/particles.hpp:294-315
  init: the field of x^0 and the half-step rollback u(-dt/2)
                                                      include/pic/simulation.hpp:56-70
Loss: 0.5 eps0 dx dy sum E^2 of the last step's field (Diagnostics ee,
include/pic/diagnostics.hpp:58-108).
"""
import numpy as np


class Case:
    def __init__(self, nx, ny, Lx, Ly, dt, qm=-1.0, eps0=1.0, B0=(0.0, 0.0, 0.0), smooth=None):
        """smooth: an optional k-space form factor s(k) [ny][nx/2 + 1] on the
        Green's function (oracle/formfactor64.py; aw_set_form_factor)."""
        self.nx, self.ny, self.Lx, self.Ly = nx, ny, Lx, Ly
        self.dx, self.dy = Lx / nx, Ly / ny
        self.dt, self.qm, self.eps0 = dt, qm, eps0
        self.B0 = np.asarray(B0, np.float64)
        kx = 2.0 * np.pi / Lx * np.arange(nx // 2 + 1)
        m = np.arange(ny)
        m = np.where(m <= ny // 2, m, m - ny)
        ky = 2.0 * np.pi / Ly * m
        KX, KY = np.meshgrid(kx, ky)                     # [ny][nkx]
        k2 = KX * KX + KY * KY
        gr = np.where(k2 > 0, 1.0 / np.where(k2 > 0, eps0 * k2, 1.0), 0.0)
        nyq = np.zeros_like(k2, bool)
        if nx % 2 == 0:
            nyq[:, nx // 2] = True
        if ny % 2 == 0:
            nyq[ny // 2, :] = True
        keep = (~nyq).astype(np.float64)
        if smooth is not None:
            gr = gr * smooth
        self.Kx = -1j * KX * gr * keep                   # E_d,k = K_d rho_k
        self.Ky = -1j * KY * gr * keep

    # ---- CIC ------------------------------------------------------------------
    def stencil(self, x, y):
        """Flat corner indices (c00, c10, c01, c11) and fractions (fx, fy)."""
        i0 = np.floor(x).astype(np.int64)
        j0 = np.floor(y).astype(np.int64)
        fx, fy = x - i0, y - j0
        i0 %= self.nx
        j0 %= self.ny
        i1, j1 = (i0 + 1) % self.nx, (j0 + 1) % self.ny
        r0, r1 = j0 * self.nx, j1 * self.nx
        return (r0 + i0, r0 + i1, r1 + i0, r1 + i1), fx, fy

    def deposit(self, st, q):
        (c00, c10, c01, c11), fx, fy = st
        m = self.ny * self.nx
        gx, gy = 1.0 - fx, 1.0 - fy
        g = np.bincount(c00, q * gx * gy, minlength=m)
        g += np.bincount(c10, q * fx * gy, minlength=m)
        g += np.bincount(c01, q * gx * fy, minlength=m)
        g += np.bincount(c11, q * fx * fy, minlength=m)
        return g.reshape(self.ny, self.nx)

    def gather(self, G, st):
        (c00, c10, c01, c11), fx, fy = st
        G = G.reshape(-1)
        gx, gy = 1.0 - fx, 1.0 - fy
        return gx * gy * G[c00] + fx * gy * G[c10] + gx * fy * G[c01] + fx * fy * G[c11]

    def gather_grad(self, G, st):
        """(dG/dx, dG/dy) of the CIC interpolant at the particles (cell units)."""
        (c00, c10, c01, c11), fx, fy = st
        G = G.reshape(-1)
        g00, g10, g01, g11 = G[c00], G[c10], G[c01], G[c11]
        ddx = (1.0 - fy) * (g10 - g00) + fy * (g11 - g01)
        ddy = (1.0 - fx) * (g01 - g00) + fx * (g11 - g10)
        return ddx, ddy

    # ---- solve and its transpose ------------------------------------------------
    def solve(self, rho):
        rk = np.fft.rfft2(rho)
        s = (self.ny, self.nx)
        return np.fft.irfft2(self.Kx * rk, s=s), np.fft.irfft2(self.Ky * rk, s=s)

    def solve_T(self, lEx, lEy):
        s = (self.ny, self.nx)
        return np.fft.irfft2(np.conj(self.Kx) * np.fft.rfft2(lEx) + np.conj(self.Ky) * np.fft.rfft2(lEy), s=s)

    # ---- Boris (u as three arrays) ------------------------------------------------
    def rot_ts(self, qmh):
        t = qmh * self.B0
        s = 2.0 * t / (1.0 + t @ t)
        return t, s

    def boris(self, u, ex, ey, qmh):
        ux, uy, uz = u
        ax, ay = qmh * ex, qmh * ey
        ux, uy = ux + ax, uy + ay
        if np.any(self.B0 != 0.0):
            (tx, ty, tz), (sx, sy, sz) = self.rot_ts(qmh)
            px, py, pz = ux + (uy * tz - uz * ty), uy + (uz * tx - ux * tz), uz + (ux * ty - uy * tx)
            ux, uy, uz = ux + (py * sz - pz * sy), uy + (pz * sx - px * sz), uz + (px * sy - py * sx)
        return ux + ax, uy + ay, uz

    def rot_T(self, lam, qmh):
        """R^T lam for the rotation u -> u + (u + u x t) x s (lam as three arrays)."""
        lx, ly, lz = lam
        if not np.any(self.B0 != 0.0):
            return lx, ly, lz
        (tx, ty, tz), (sx, sy, sz) = self.rot_ts(qmh)
        cx, cy, cz = ly * sz - lz * sy, lz * sx - lx * sz, lx * sy - ly * sx      # lam x s
        return (lx - cx + (cy * tz - cz * ty), ly - cy + (cz * tx - cx * tz), lz - cz + (cx * ty - cy * tx))

    # ---- forward / backward ----------------------------------------------------------
    def forward(self, x, y, u, w, nsteps, keep=True):
        """Initial state (x, y in cell units, u [n][3], w) -> (loss, trajectory, q)."""
        x, y = np.array(x, np.float64), np.array(y, np.float64)
        u = tuple(np.array(u[:, d], np.float64) for d in range(3))
        q = self.qm / (self.dx * self.dy) * np.asarray(w, np.float64)
        qmh = self.qm * 0.5 * self.dt
        qmh_b = self.qm * 0.5 * (-0.5 * self.dt)
        st = self.stencil(x, y)
        ex, ey = self.solve(self.deposit(st, q))
        u = self.boris(u, self.gather(ex, st), self.gather(ey, st), qmh_b)
        traj = []
        for _ in range(nsteps):
            st = self.stencil(x, y)
            ex, ey = self.solve(self.deposit(st, q))
            if keep:
                traj.append((x.copy(), y.copy(), ex, ey))
            u = self.boris(u, self.gather(ex, st), self.gather(ey, st), qmh)
            x = np.mod(x + u[0] * (self.dt / self.dx), self.nx)
            y = np.mod(y + u[1] * (self.dt / self.dy), self.ny)
        loss = 0.5 * self.eps0 * self.dx * self.dy * float(np.sum(ex * ex + ey * ey))
        return loss, traj, q

    def gradient(self, x, y, u, w, nsteps):
        """(loss, dloss/du0 [n][3]) by the discrete adjoint of forward()."""
        loss, traj, q = self.forward(x, y, u, w, nsteps)
        n = len(q)
        qmh = self.qm * 0.5 * self.dt
        qmh_b = self.qm * 0.5 * (-0.5 * self.dt)
        cx, cy = self.dt / self.dx, self.dt / self.dy
        lx, ly = np.zeros(n), np.zeros(n)
        lu = (np.zeros(n), np.zeros(n), np.zeros(n))
        ext = self.eps0 * self.dx * self.dy
        for s in range(nsteps - 1, -1, -1):
            xs, ys, ex, ey = traj[s]
            st = self.stencil(xs, ys)
            lu3 = (lu[0] + cx * lx, lu[1] + cy * ly, lu[2])
            lu1 = self.rot_T(lu3, qmh)
            lEx = qmh * (lu3[0] + lu1[0])
            lEy = qmh * (lu3[1] + lu1[1])
            dxx, dxy = self.gather_grad(ex, st)
            dyx, dyy = self.gather_grad(ey, st)
            lx = lx + lEx * dxx + lEy * dyx
            ly = ly + lEx * dxy + lEy * dyy
            lu = lu1
            gEx = self.deposit(st, lEx)
            gEy = self.deposit(st, lEy)
            if s == nsteps - 1:
                gEx = gEx + ext * ex
                gEy = gEy + ext * ey
            lrho = self.solve_T(gEx, gEy)
            ddx, ddy = self.gather_grad(lrho, st)
            lx = lx + q * ddx
            ly = ly + q * ddy
        return loss, np.stack(self.rot_T(lu, qmh_b), axis=1)


def loss_at(case, x, y, u, w, nsteps):
    return case.forward(x, y, u, w, nsteps, keep=False)[0]


def central_difference(case, x, y, u, w, nsteps, direction, h):
    """(L(u + h d) - L(u - h d)) / 2h in float64."""
    lp = loss_at(case, x, y, u + h * direction, w, nsteps)
    lm = loss_at(case, x, y, u - h * direction, w, nsteps)
    return (lp - lm) / (2.0 * h)
