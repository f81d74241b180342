"""Unit-sphere angular tables for 2D and 3D solves: the Carlson level-symmetric quadrature, real
(full- and half-range) spherical harmonics and the Galerkin bases built from them.

Each function restates the cited Radiant.jl function with the same arithmetic.
"""
from __future__ import annotations

import math

import numpy as np


def newton_bisection(f, dfdx, x1: float, x2: float, eps0: float = np.finfo(float).eps, nmax: int = 100) -> float:
    """Safeguarded Newton iteration inside a bracket (src/tools/newton_bisection.jl)."""
    f1, f2 = f(x1), f(x2)
    if f1 * f2 > 0.0:
        raise ValueError("Root must be bracketed: f(x1) and f(x2) must have opposite signs.")
    if f1 == 0.0:
        return x1
    if f2 == 0.0:
        return x2
    xl, xh = (x1, x2) if f1 < 0 else (x2, x1)
    rts = 0.5 * (x1 + x2)
    dxold = abs(x2 - x1)
    dx = dxold
    f_rts, df_rts = f(rts), dfdx(rts)
    for _ in range(nmax):
        if ((rts - xh) * df_rts - f_rts) * ((rts - xl) * df_rts - f_rts) > 0.0 or abs(2.0 * f_rts) > abs(dxold * df_rts):
            dxold = dx
            dx = 0.5 * (xh - xl)
            rts = xl + dx
        else:
            dxold = dx
            dx = f_rts / df_rts
            rts -= dx
        if abs(dx) < eps0:
            return rts
        f_rts, df_rts = f(rts), dfdx(rts)
        if f_rts < 0.0:
            xl = rts
        else:
            xh = rts
    raise RuntimeError(f"Maximum number of iterations ({nmax}) exceeded in newton_bisection.")


def carlson(N: int):
    """Carlson level-symmetric quadrature, N(N+2) directions on the unit sphere
    (src/tools/carlson.jl:20-94). Returns ([mu, eta, xi], w) with Σw = 4π."""
    if N < 2 or N % 2 != 0:
        raise ValueError("Carlson quadrature available for even N ≥ 2.")
    h = N // 2
    M = N * (N + 2)
    mu, eta, xi, w = np.zeros(M), np.zeros(M), np.zeros(M), np.zeros(M)
    wn = np.array([4 * (N - 2 * n + 2) / (N * (N + 2)) for n in range(1, h + 1)])
    mun_m = np.array([1 - (N - 2 * n + 2) * (N - 2 * n + 4) / (N * (N + 2)) for n in range(1, h + 1)])
    mun0 = np.array([1 - (N - 2 * n + 2) ** 2 / (N * (N + 2)) for n in range(1, h + 1)])
    if N == 2:
        mun = np.array([1 / math.sqrt(3)])
    else:
        f = lambda x: 1 / 3 - float(np.sum(wn * (mun0 + x * mun_m) ** 2))
        dfdx = lambda x: -float(np.sum(2 * wn * mun_m * (mun0 + x * mun_m)))
        x = newton_bisection(f, dfdx, 1.0, -1.0)
        mun = np.array([mun0[n] + x * mun_m[n] for n in range(h)])
    w0 = 1 / (N * (N + 2))
    if N == 2:
        A = 1.0
    else:
        def g(A):
            s = 0.0
            for n in range(1, h + 1):
                s += (math.pi / 2 * wn[n - 1] * mun[n - 1] - 4 * math.pi * w0 / math.sqrt(2) * math.sin(math.pi * A / 4)
                      * math.sqrt(1 - mun[n - 1] ** 2) / math.sin(math.pi * A / (2 * N - 4 * n + 4)))
            return s

        def dgdA(A):
            s = 0.0
            for n in range(1, h + 1):
                a = math.pi * A / (2 * N - 4 * n + 4)
                r = math.sqrt(1 - mun[n - 1] ** 2)
                s += -4 * math.pi * w0 * math.sqrt(2) * math.pi / 8 * (
                    math.cos(math.pi * A / 4) * r / math.sin(a)
                    - 2 * math.sin(math.pi * A / 4) * r * math.cos(a) / math.sin(a) ** 2 / (N - 2 * n + 2))
            return s

        A = newton_bisection(g, dgdA, 1 / 2, 2.0)
    i = 0
    s = [(1, 1, 1), (1, 1, -1), (1, -1, 1), (1, -1, -1), (-1, 1, 1), (-1, 1, -1), (-1, -1, 1), (-1, -1, -1)]
    for t in range(8):
        for n in range(1, h + 1):
            for m in range(1, h - n + 2):
                phi = math.pi / 2 * ((2 * m - 1) / (N - 2 * n + 2) * A + (1 - A) / 2)
                mu[i] = s[t][0] * mun[n - 1]
                eta[i] = s[t][1] * math.sqrt(1 - mu[i] ** 2) * math.cos(phi)
                xi[i] = s[t][2] * math.sqrt(1 - mu[i] ** 2) * math.sin(phi)
                w[i] = w0
                i += 1
    return [mu, eta, xi], 4 * math.pi * w


def factorial_factor(num, den, exp_terms=()):
    """exp(Σ log n! − Σ log d! + Σ m·log x) (src/tools/factorial_factor.jl)."""
    fac = 0.0
    for n in num:
        for i in range(1, n + 1):
            fac += math.log(i)
    for n in den:
        for i in range(1, n + 1):
            fac -= math.log(i)
    for x, m in exp_terms:
        if m == 0:  # Julia's `m ≈ 0` against zero is exact equality
            continue
        if x == 0:
            return 0.0 if m > 0 else math.inf
        fac += m * math.log(x)
    return math.exp(fac)


def jacobi_polynomials_up_to_L(L: int, a: int, b: int, x: float) -> np.ndarray:
    """P_l^(α,β)(x), l = 0..L (src/tools/jacobi_polynomials.jl)."""
    P = np.zeros(L + 1)
    if x == 1:
        for l in range(L + 1):
            P[l] = factorial_factor([l + a], [l, a])
    elif x == -1:
        for l in range(L + 1):
            P[l] = (-1) ** l * factorial_factor([l + b], [l, b])
    else:
        P[0] = 1.0
        if L >= 1:
            P[1] = (a + 1) + 0.5 * (a + b + 2) * (x - 1)
        for l in range(2, L + 1):
            if l < 125:
                P[l] = ((2 * l + a + b - 1) * ((2 * l + a + b) * (2 * l + a + b - 2) * x + a ** 2 - b ** 2) * P[l - 1]
                        - (2 * (l + a - 1) * (l + b - 1) * (2 * l + a + b)) * P[l - 2]) / (2 * l * (l + a + b) * (2 * l + a + b - 2))
            else:
                th = math.acos(x)
                kth = 1 / (math.sqrt(math.pi) * math.sin(0.5 * th) ** (a + 0.5) * math.cos(0.5 * th) ** (b + 0.5))
                Nn = l + 0.5 * (a + b + 1)
                gam = -0.5 * math.pi * (a + 0.5)
                P[l] = 1 / math.sqrt(l) * kth * math.cos(Nn * th + gam)
    return P


def _assoc_legendre(L: int, x: float, half: bool):
    """Plm[l][m] as in real_spherical_harmonics.jl:52-103 (x = μ) and :104-151 (x = 2μ−1)."""
    Plm = [np.zeros(l + 1) for l in range(L + 1)]
    mu = x
    arg = 2 * mu - 1 if half else mu
    if mu == -1 or mu == 1:
        Pl = jacobi_polynomials_up_to_L(L, 0, 0, arg)
        for l in range(L + 1):
            Plm[l][0] = Pl[l]
    else:
        for m in range(L + 1):
            Pl = jacobi_polynomials_up_to_L(L - m, m, m, arg)
            for l in range(m, L + 1):
                Plm[l][m] = factorial_factor([l + m], [l], [(2, -m), (1 - arg ** 2, m / 2)]) * Pl[l - m]
    return Plm


def real_spherical_harmonics_up_to_L(L: int, mu: float, phi: float):
    """R_lm(μ, ϕ), l = 0..L, m = -l..l (real_spherical_harmonics.jl:52-103)."""
    if not (-1 <= mu <= 1):
        raise ValueError("Invalid direction cosine (should be between -1 and 1).")
    Plm = _assoc_legendre(L, mu, False)
    R = [np.zeros(2 * l + 1) for l in range(L + 1)]
    for l in range(L + 1):
        for m in range(-l, l + 1):
            Tm = math.cos(m * phi) if m >= 0 else math.sin(abs(m) * phi)
            C = math.sqrt((2 - (m == 0)) * factorial_factor([l - abs(m)], [l + abs(m)]))
            R[l][l + m] = C * Plm[l][abs(m)] * Tm
    return R


def real_half_range_spherical_harmonics_up_to_L(L: int, mu: float, phi: float):
    """Half-range real spherical harmonics (real_spherical_harmonics.jl:104-151)."""
    if not (0 <= mu <= 1):
        raise ValueError("Invalid direction cosine (should be between 0 and 1).")
    Plm = _assoc_legendre(L, mu, True)
    Y = [np.zeros(2 * l + 1) for l in range(L + 1)]
    for l in range(L + 1):
        for m in range(-l, l + 1):
            Tm = math.cos(m * phi) if m >= 0 else math.sin(abs(m) * phi)
            C = math.sqrt((2 - (m == 0)) / (2 * math.pi) * (2 * l + 1) * factorial_factor([l - abs(m)], [l + abs(m)]))
            Y[l][l + m] = C * Plm[l][abs(m)] * Tm
    return Y


def angular_matrix_gram_schmidt(Nd: int, L: int, Rlm, w, Qdims: int, g_type: int = 1):
    """Select Nd independent harmonics by Gram-Schmidt and build the square Galerkin pair
    (angular_polynomial_basis.jl:465-548). Returns ok, Np, Mn, Dn, pl, pm."""
    pl = np.zeros(Nd, dtype=np.int64)
    pm = np.zeros(Nd, dtype=np.int64)
    Mn = np.zeros((Nd, Nd))
    Dn = np.zeros((Nd, Nd))
    u = np.zeros((Nd, Nd))
    vec0 = np.array([Rlm[n2][0][0] for n2 in range(Nd)])
    nrm0 = math.sqrt(float(np.sum(vec0 * vec0)))
    for n in range(Nd):
        if g_type == 1:
            Dn[0, n] = w[n] * Rlm[n][0][0]
        elif g_type == 2:
            Mn[n, 0] = 1 / (4 * math.pi) * Rlm[n][0][0]
        elif g_type == 3:
            Mn[n, 0] = Rlm[n][0][0]
        u[n, 0] = Rlm[n][0][0] / nrm0
    i = 1
    for l in range(1, L + 1):
        m_min = 0 if Qdims == 2 else -l
        for m in range(m_min, l + 1):
            vec = np.array([Rlm[n2][l][m + l] for n2 in range(Nd)])
            S = np.zeros(Nd)
            for k in range(i):
                S += float(np.sum(u[:, k] * vec)) * u[:, k]
            vk = vec - S
            nv = math.sqrt(float(np.sum(vk * vk)))
            if nv > 1e-5:
                i += 1
                u[:, i - 1] = vk / nv
                for n in range(Nd):
                    if g_type == 1:
                        Dn[i - 1, n] = w[n] * Rlm[n][l][m + l]
                    elif g_type == 2:
                        Mn[n, i - 1] = (2 * l + 1) / (4 * math.pi) * Rlm[n][l][m + l]
                    elif g_type == 3:
                        Mn[n, i - 1] = Rlm[n][l][m + l]
                pl[i - 1] = l
                pm[i - 1] = m
            if Nd == i:
                break
        if Nd == i:
            break
    if i < Nd:
        return False, Nd, np.zeros((Nd, Nd)), np.zeros((Nd, Nd)), pl, pm
    if g_type == 1:
        Mn = np.linalg.inv(Dn)
    else:
        Dn = np.linalg.inv(Mn)
    return True, Nd, Mn, Dn, pl, pm


def angular_polynomial_basis_sphere(Om, w, L: int, btype: str, Qdims: int):
    """Np, Mn, Dn, pl, pm for Qdims = 2 or 3 (angular_polynomial_basis.jl:51-179)."""
    from .tables import galerkin_minimum_order

    mu, eta, xi = (np.asarray(a, dtype=float) for a in Om)
    Nd = len(w)
    Lb = max(L, galerkin_minimum_order(Nd, Qdims)) if btype in ("galerkin-m", "galerkin-d") else L
    phi = np.arctan2(xi, eta)
    Rlm = [real_spherical_harmonics_up_to_L(Lb, float(mu[n]), float(phi[n])) for n in range(Nd)]
    if btype == "standard":
        Np = (L + 1) * (L + 2) // 2 if Qdims == 2 else (L + 1) ** 2
        pl = np.zeros(Np, dtype=np.int64)
        pm = np.zeros(Np, dtype=np.int64)
        Mn = np.zeros((Nd, Np))
        Dn = np.zeros((Np, Nd))
        li = 0
        for l in range(L + 1):
            for m in range(-l, l + 1):
                if Qdims == 2 and (l + m) % 2 == 1:
                    continue
                pl[li], pm[li] = l, m
                for n in range(Nd):
                    Mn[n, li] = (2 * l + 1) / (4 * math.pi) * Rlm[n][l][m + l]
                    Dn[li, n] = w[n] * Rlm[n][l][m + l]
                li += 1
        return Np, Mn, Dn, pl, pm
    if btype in ("galerkin-d", "galerkin-m"):
        g_type = 1 if btype == "galerkin-d" else 2
        Lg = Lb
        ok, Np, Mn, Dn, pl, pm = angular_matrix_gram_schmidt(Nd, Lg, Rlm, w, Qdims, g_type)
        while not ok:
            Lg += 1
            if Lg > Lb + Nd + 10:
                raise RuntimeError(f"Galerkin (Qdims={Qdims}): unable to find {Nd} independent spherical harmonics")
            Rlm = [real_spherical_harmonics_up_to_L(Lg, float(mu[n]), float(phi[n])) for n in range(Nd)]
            ok, Np, Mn, Dn, pl, pm = angular_matrix_gram_schmidt(Nd, Lg, Rlm, w, Qdims, g_type)
        return Np, Mn, Dn, pl, pm
    raise ValueError("Unknown method.")


def surface_basis_sphere_face(Om, w, L: int, btype: str, Qdims: int, surface: str):
    """Half-range basis of one face of a 2D/3D geometry (angular_polynomial_basis.jl:249-436)."""
    from .tables import galerkin_minimum_order

    mu, eta, xi = (np.asarray(a, dtype=float) for a in Om)
    s = surface.upper()
    if s == "X-":
        idx = np.nonzero(mu > 0)[0]; mup = mu[idx]; ph = np.arctan2(xi, eta)
    elif s == "X+":
        idx = np.nonzero(mu < 0)[0]; mup = -mu[idx]; ph = np.arctan2(xi, eta)
    elif s == "Y-":
        idx = np.nonzero(eta > 0)[0]; mup = eta[idx]; ph = np.arctan2(mu, xi)
    elif s == "Y+":
        idx = np.nonzero(eta < 0)[0]; mup = -eta[idx]; ph = np.arctan2(mu, xi)
    elif s == "Z-":
        idx = np.nonzero(xi > 0)[0]; mup = xi[idx]; ph = np.arctan2(eta, mu)
    elif s == "Z+":
        idx = np.nonzero(xi < 0)[0]; mup = -xi[idx]; ph = np.arctan2(eta, mu)
    else:
        raise ValueError("Unknown surface for 3D angular domain.")
    Ndp = len(idx)
    php = ph[idx]
    wp = np.asarray(w)[idx]
    Lb = max(L, galerkin_minimum_order(Ndp, Qdims)) if btype in ("galerkin-m", "galerkin-d") else L
    psi = [real_half_range_spherical_harmonics_up_to_L(Lb, abs(float(mup[k])), float(php[k])) for k in range(Ndp)]
    Nd = len(mu)
    n_to_np = np.zeros(Nd, dtype=np.int64)
    for k, n in enumerate(idx):
        n_to_np[n] = k + 1
    if btype == "standard":
        Np = (L + 1) * (L + 2) // 2 if Qdims == 2 else (L + 1) ** 2
        pl = np.zeros(Np, dtype=np.int64)
        pm = np.zeros(Np, dtype=np.int64)
        Mn = np.zeros((Ndp, Np))
        Dn = np.zeros((Np, Ndp))
        li = 0
        for l in range(L + 1):
            for m in range(-l, l + 1):
                if Qdims == 2 and (l + m) % 2 == 1:
                    continue
                pl[li], pm[li] = l, m
                for k in range(Ndp):
                    Mn[k, li] = psi[k][l][l + m]
                    Dn[li, k] = wp[k] * psi[k][l][l + m]
                li += 1
    elif btype in ("galerkin-d", "galerkin-m"):
        g_type = 1 if btype == "galerkin-d" else 3
        Lg = Lb
        ok, Np, Mn, Dn, pl, pm = angular_matrix_gram_schmidt(Ndp, Lg, psi, wp, Qdims, g_type)
        while not ok:
            Lg += 1
            if Lg > Lb + Ndp + 10:
                raise RuntimeError("Surface Galerkin: unable to find independent half-range harmonics")
            psi = [real_half_range_spherical_harmonics_up_to_L(Lg, abs(float(mup[k])), float(php[k])) for k in range(Ndp)]
            ok, Np, Mn, Dn, pl, pm = angular_matrix_gram_schmidt(Ndp, Lg, psi, wp, Qdims, g_type)
    else:
        raise ValueError("Unknown method.")
    return Np, Mn, Dn, idx + 1, n_to_np, pl, pm


def surface_source_moments(Om, w, L: int, btype: str, Qdims: int, surface: str, direction, intensity: float = 1.0):
    """Half-range moments of a monodirectional beam through one face (surface_source.jl:97-128
    for SN): returns (moments[Np], pl, pm)."""
    Np, _, _, _, _, pl, pm = surface_basis_sphere_face(Om, w, L, btype, Qdims, surface)
    mus, etas, xis = direction
    phis = math.atan2(xis, etas)
    Lmax = int(np.max(pl))
    ps = real_half_range_spherical_harmonics_up_to_L(Lmax, abs(mus), phis)
    q = np.array([intensity * ps[pl[p]][pl[p] + pm[p]] for p in range(Np)])
    return q, pl, pm
