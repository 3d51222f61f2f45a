"""Method of moving asymptotes, one subproblem step (oracle, test only).

The reference calls ``mmapy.mmasub`` (mmapy==0.3.1, a third-party package that
is neither vendored in the reference nor installed here) from
deep_frame/topology_optimizers.py:40,61-63 with a0 = 1, a = 0, c = 1e4, d = 1
and f, g scaled by 100.  MMA numerics are therefore parity-unpinned; this
module restates K. Svanberg's published method -- "The method of moving
asymptotes" (IJNME 24, 1987) and "MMA and GCMMA, two methods for nonlinear
optimization" (KTH, 2007), sections on the asymptote update, the move limits,
the convex approximations and the primal-dual interior-point subproblem
solver -- in NumPy.  The CUDA implementation (tf_mma_step) follows the same
sequence of operations and is checked against it.
"""
import numpy as np

DEFAULTS = {"move": 0.5, "asyinit": 0.5, "asydecr": 0.7, "asyincr": 1.2, "asymin": 0.01, "asymax": 10.0,
            "raa0": 1e-5, "albefa": 0.1, "epsimin": 1e-7}


def asymptotes(iteration, x, xmin, xmax, xold1, xold2, low, upp, s):
    span = xmax - xmin
    if iteration <= 2:
        return x - s["asyinit"] * span, x + s["asyinit"] * span
    trend = (x - xold1) * (xold1 - xold2)
    factor = np.ones_like(x)
    factor[trend > 0] = s["asyincr"]
    factor[trend < 0] = s["asydecr"]
    low = x - factor * (xold1 - low)
    upp = x + factor * (upp - xold1)
    low = np.clip(low, x - s["asymax"] * span, x - s["asymin"] * span)
    upp = np.clip(upp, x + s["asymin"] * span, x + s["asymax"] * span)
    return low, upp


def approximation(x, xmin, xmax, low, upp, df0dx, fval, dfdx, s):
    span = np.maximum(xmax - xmin, 1e-5)
    alfa = np.maximum(np.maximum(low + s["albefa"] * (x - low), x - s["move"] * (xmax - xmin)), xmin)
    beta = np.minimum(np.minimum(upp - s["albefa"] * (upp - x), x + s["move"] * (xmax - xmin)), xmax)
    ux1, xl1 = upp - x, x - low
    ux2, xl2 = ux1 ** 2, xl1 ** 2
    p0 = np.maximum(df0dx, 0.0)
    q0 = np.maximum(-df0dx, 0.0)
    pq0 = 0.001 * (p0 + q0) + s["raa0"] / span
    p0 = (p0 + pq0) * ux2
    q0 = (q0 + pq0) * xl2
    P = np.maximum(dfdx, 0.0)
    Q = np.maximum(-dfdx, 0.0)
    PQ = 0.001 * (P + Q) + s["raa0"] / span[None, :]
    P = (P + PQ) * ux2[None, :]
    Q = (Q + PQ) * xl2[None, :]
    b = P @ (1.0 / ux1) + Q @ (1.0 / xl1) - fval
    return alfa, beta, p0, q0, P, Q, b


def subsolve(m, n, epsimin, low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d, trace=None):
    """Primal-dual Newton iterations on the perturbed KKT system of the MMA subproblem."""
    x = 0.5 * (alfa + beta)
    y = np.ones(m)
    z = 1.0
    lam = np.ones(m)
    xsi = np.maximum(1.0 / (x - alfa), 1.0)
    eta = np.maximum(1.0 / (beta - x), 1.0)
    mu = np.maximum(np.ones(m), 0.5 * c)
    zet = 1.0
    s = np.ones(m)
    epsi = 1.0
    while epsi > epsimin:
        def residual(x, y, z, lam, xsi, eta, mu, zet, s):
            ux1, xl1 = upp - x, x - low
            plam = p0 + P.T @ lam
            qlam = q0 + Q.T @ lam
            gvec = P @ (1.0 / ux1) + Q @ (1.0 / xl1)
            dpsidx = plam / ux1 ** 2 - qlam / xl1 ** 2
            parts = [dpsidx - xsi + eta, c + d * y - mu - lam, [a0 - zet - a @ lam], gvec - a * z - y + s - b,
                     xsi * (x - alfa) - epsi, eta * (beta - x) - epsi, mu * y - epsi, [zet * z - epsi], lam * s - epsi]
            r = np.concatenate([np.atleast_1d(np.asarray(p, dtype=float)) for p in parts])
            return np.sqrt(r @ r), np.max(np.abs(r))
        norm, rmax = residual(x, y, z, lam, xsi, eta, mu, zet, s)
        inner = 0
        while rmax > 0.9 * epsi and inner < 200:
            inner += 1
            ux1, xl1 = upp - x, x - low
            ux2, xl2 = ux1 ** 2, xl1 ** 2
            ux3, xl3 = ux1 * ux2, xl1 * xl2
            uxinv1, xlinv1 = 1.0 / ux1, 1.0 / xl1
            plam = p0 + P.T @ lam
            qlam = q0 + Q.T @ lam
            gvec = P @ uxinv1 + Q @ xlinv1
            GG = P / ux2[None, :] - Q / xl2[None, :]
            dpsidx = plam / ux2 - qlam / xl2
            delx = dpsidx - epsi / (x - alfa) + epsi / (beta - x)
            dely = c + d * y - lam - epsi / y
            delz = a0 - a @ lam - epsi / z
            dellam = gvec - a * z - y - b + epsi / lam
            diagx = 2 * (plam / ux3 + qlam / xl3) + xsi / (x - alfa) + eta / (beta - x)
            diagy = d + mu / y
            diaglamyi = s / lam + 1.0 / diagy
            blam = dellam + dely / diagy - GG @ (delx / diagx)
            alam = np.diag(diaglamyi) + (GG / diagx[None, :]) @ GG.T
            aa = np.zeros((m + 1, m + 1))
            aa[:m, :m] = alam
            aa[:m, m] = a
            aa[m, :m] = a
            aa[m, m] = -zet / z
            sol = np.linalg.solve(aa, np.concatenate([blam, [delz]]))
            dlam, dz = sol[:m], sol[m]
            dx = -delx / diagx - (GG.T @ dlam) / diagx
            dy = -dely / diagy + dlam / diagy
            dxsi = -xsi + epsi / (x - alfa) - xsi * dx / (x - alfa)
            deta = -eta + epsi / (beta - x) + eta * dx / (beta - x)
            dmu = -mu + epsi / y - mu * dy / y
            dzet = -zet + epsi / z - zet * dz / z
            ds = -s + epsi / lam - s * dlam / lam
            stm = max(np.max(-1.01 * np.concatenate([dy / y, [dz / z], dlam / lam, dxsi / xsi, deta / eta, dmu / mu, [dzet / zet], ds / s])),
                      np.max(-1.01 * dx / (x - alfa)), np.max(1.01 * dx / (beta - x)), 1.0)
            step = 1.0 / stm
            old = (x, y, z, lam, xsi, eta, mu, zet, s)
            tries, new_norm = 0, 2 * norm
            while new_norm > norm and tries < 50:
                tries += 1
                x, y, z, lam, xsi, eta, mu, zet, s = (o + step * dd for o, dd in zip(old, (dx, dy, dz, dlam, dxsi, deta, dmu, dzet, ds)))
                new_norm, new_max = residual(x, y, z, lam, xsi, eta, mu, zet, s)
                step /= 2
            norm, rmax = new_norm, new_max
            if trace is not None:
                trace.append((epsi, inner, tries, norm, rmax))
        epsi *= 0.1
    return x, y, z, lam, xsi, eta, mu, zet, s


def mmasub(m, n, iteration, xval, xmin, xmax, xold1, xold2, f0val, df0dx, fval, dfdx, low, upp, a0, a, c, d, **settings):
    """One MMA step.  Vectors are 1-D ([n] or [m]); dfdx is [m, n].  Returns (x, y, z, lam, low, upp)."""
    s = {**DEFAULTS, **settings}
    x = np.asarray(xval, dtype=float).ravel()
    xmin, xmax = np.broadcast_to(np.asarray(xmin, dtype=float).ravel(), x.shape), np.broadcast_to(np.asarray(xmax, dtype=float).ravel(), x.shape)
    low, upp = asymptotes(iteration, x, xmin, xmax, np.asarray(xold1, float).ravel(), np.asarray(xold2, float).ravel(),
                          np.asarray(low, float).ravel(), np.asarray(upp, float).ravel(), s)
    alfa, beta, p0, q0, P, Q, b = approximation(x, xmin, xmax, low, upp, np.asarray(df0dx, float).ravel(),
                                                np.asarray(fval, float).ravel(), np.asarray(dfdx, float).reshape(m, n), s)
    xn, y, z, lam, *_ = subsolve(m, n, s["epsimin"], low, upp, alfa, beta, p0, q0, P, Q, float(a0),
                                  np.asarray(a, float).ravel(), b, np.asarray(c, float).ravel(), np.asarray(d, float).ravel())
    return xn, y, z, lam, low, upp
