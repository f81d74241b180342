"""Host-side tables of the SN solve: quadratures, angular bases, closure weights, and the
angular Fokker-Planck matrix.

These are the arrays Radiant.jl's ``compute_flux(::SN)`` builds once per solve before its
group loop (src/particle_transport/sn_flux.jl:44-106). They are small and built on the host,
exactly as in the reference; every function below restates the cited reference function
with the same arithmetic so that indexing and table layout match it.
"""
from __future__ import annotations

import math

import numpy as np

# --------------------------------------------------------------------------------------
# Legendre polynomials (src/tools/legendre_polynomials.jl)
# --------------------------------------------------------------------------------------


def legendre_polynomials_up_to_L(L: int, x: float) -> np.ndarray:
    """P_0..P_L at x by Bonnet's recursion (legendre_polynomials.jl:67-89)."""
    if L < 0:
        raise ValueError("Legendre order is greater or equal to zero.")
    if not (-1.0 <= x <= 1.0):
        raise ValueError("Invalid x value (should be between -1 and 1).")
    Pl = np.zeros(L + 1)
    if x == 1:
        Pl[:] = 1.0
    elif x == -1:
        Pl[:] = [(-1.0) ** l for l in range(L + 1)]
    else:
        Pl[0] = 1.0
        if L >= 1:
            Pl[1] = x
        for l in range(2, L + 1):
            Pl[l] = ((2 * l - 1) * x * Pl[l - 1] - (l - 1) * Pl[l - 2]) / l
    return Pl


def half_range_legendre_polynomials_up_to_L(L: int, x: float) -> np.ndarray:
    """sqrt(2l+1)·P_l(2x-1) (legendre_polynomials.jl:101-103)."""
    return np.sqrt(2.0 * np.arange(L + 1) + 1.0) * legendre_polynomials_up_to_L(L, 2.0 * x - 1.0)


# --------------------------------------------------------------------------------------
# Quadratures (src/tools/quadrature.jl, gauss_legendre.jl, carlson.jl)
# --------------------------------------------------------------------------------------


def gauss_legendre(N: int):
    """Gauss-Legendre nodes/weights: asymptotic first guess then Newton on Bonnet's
    recursion to machine precision (src/tools/gauss_legendre.jl:18-74)."""
    x = np.zeros(N)
    for i in range(1, N // 2 + 1):
        phi = math.pi / 2 * (4 * i - 1) / (2 * N + 1)
        x[i - 1] = (1 - (N - 1) / (8 * N ** 3) - 1 / (384 * N ** 4) * (39 - 28 / (math.sin(phi) ** 2))) * math.cos(phi)
        x[N - i] = -x[i - 1]
    w = np.zeros(N)
    dPdx = 0.0
    eps = np.finfo(float).eps
    for i in range(N):
        xi = float(x[i])
        xold = 2.0
        while abs(xi - xold) > eps:
            xold = xi
            P0, P1 = 1.0, xi
            for n in range(2, N + 1):
                Pn = ((2 * n - 1) * xi * P1 - (n - 1) * P0) / n
                P0, P1 = P1, Pn
            dPdx = N * (P0 - xi * P1) / (1 - xi ** 2)
            xi -= P1 / dPdx
        x[i] = xi
        w[i] = 2 / ((1 - xi ** 2) * dPdx ** 2)
    if len(set(x.tolist())) != N:
        raise ValueError(f"Unable to build Lobatto quadrature at order N = {N}.")
    return x, w


def gauss_lobatto(N: int):
    """Gauss-Lobatto nodes/weights: end points ±1, interior nodes the zeros of P'_(N−1) by Newton
    from the Chebyshev-Lobatto guess (src/tools/gauss_lobatto.jl), nodes in decreasing order."""
    x = np.cos(np.pi * np.arange(N) / (N - 1))
    w = np.zeros(N)
    w[0] = w[-1] = 2 / (N * (N - 1))
    eps = np.finfo(float).eps
    for i in range(1, N - 1):
        xi, xold = float(x[i]), 2.0
        P1 = 0.0
        while abs(xi - xold) > eps:
            xold = xi
            P0, P1 = 1.0, xi
            for n in range(2, N):
                Pn = ((2 * n - 1) * xi * P1 - (n - 1) * P0) / n
                P0, P1 = P1, Pn
            dPdx = N * (P0 - xi * P1) / (1 - xi ** 2)
            d2 = (2 * xi * dPdx - N * (N + 1) * P1) / (1 - xi ** 2)
            xi -= dPdx / d2
        x[i] = xi
        w[i] = 2 / (N * (N - 1) * P1 ** 2)
    return x, w


def gauss_legendre_chebychev(N: int):
    """Product quadrature: N Gauss-Legendre polar levels (ascending μ) × 2N equally spaced
    azimuths ϕ = π(m − 1/2)/N, weight w_n·π/N (src/tools/gauss_legendre_chebychev.jl)."""
    mun, wn = gauss_legendre(N)
    idx = np.argsort(mun, kind="stable")
    mun, wn = mun[idx], wn[idx]
    mu, eta, xi, w = (np.zeros(2 * N * N) for _ in range(4))
    i = 0
    for n in range(N):
        for m in range(1, 2 * N + 1):
            phi = math.pi / N * (m - 0.5)
            s = math.sqrt(1 - mun[n] ** 2)
            mu[i], eta[i], xi[i], w[i] = mun[n], s * math.cos(phi), s * math.sin(phi), wn[n] * math.pi / N
            i += 1
    return [mu, eta, xi], w


def quadrature(N: int, qtype: str, Ndims: int = 1, Qdims: int | None = None):
    """Directions and weights (src/tools/quadrature.jl:19-58). 1D returns (mu, w); the
    unit-sphere types return ([mu, eta, xi], w), folded onto ξ ≥ 0 when Qdims == 2."""
    if Qdims is None:
        Qdims = Ndims
    if qtype == "gauss-legendre" and Ndims == 1:
        Om, w = gauss_legendre(N)
    elif qtype == "gauss-lobatto" and Ndims == 1:
        Om, w = gauss_lobatto(N)
    elif qtype == "gauss-legendre-chebychev":
        Om, w = gauss_legendre_chebychev(N)
    elif qtype == "carlson":
        from .sphere import carlson

        Om, w = carlson(N)
    else:
        raise ValueError(f"Unknown {qtype} quadrature in {Ndims}D geometry.")
    if Qdims == 2:
        mu, eta, xi = Om
        cond = xi >= 0
        w0 = w.copy()
        Nd = len(w)
        for i in range(Nd):
            if not cond[i]:
                eps_xi = np.abs(mu[i] - mu) ** 2 + np.abs(eta[i] - eta) ** 2 + np.abs(xi[i] + xi) ** 2
                w0[int(np.argmin(eps_xi))] += w0[i]
        w = w0[cond]
        Om = [mu[cond], eta[cond], xi[cond]]
    return Om, w


# --------------------------------------------------------------------------------------
# Angular bases (src/particle_transport/angular_polynomial_basis.jl)
# --------------------------------------------------------------------------------------


def galerkin_minimum_order(Nd: int, Qdims: int) -> int:
    """angular_polynomial_basis.jl:9-17."""
    if Qdims == 1:
        return Nd - 1
    n = 0
    while True:
        count = (n + 1) * (n + 2) // 2 if Qdims == 2 else (n + 1) ** 2
        if count >= Nd:
            return n
        n += 1


def angular_polynomial_basis(Om, w, L: int, btype: str, Qdims: int):
    """Np, Mn[Nd,Np], Dn[Np,Nd], pl, pm (angular_polynomial_basis.jl:51-179)."""
    if Qdims == 1:
        mu = np.asarray(Om[0], dtype=float)
        Nd = len(mu)
        Lb = max(L, galerkin_minimum_order(Nd, 1)) if btype in ("galerkin-m", "galerkin-d") else L
        Pl = [legendre_polynomials_up_to_L(Lb, float(mu[n])) for n in range(Nd)]
        if btype == "standard":
            Np = L + 1
            pl = np.arange(Np, dtype=np.int64)
            Mn = np.zeros((Nd, Np)); Dn = np.zeros((Np, Nd))
            for l in range(L + 1):
                for n in range(Nd):
                    Mn[n, l] = (2 * l + 1) / 2 * Pl[n][l]
                    Dn[l, n] = w[n] * Pl[n][l]
        elif btype == "galerkin-m":
            Np = Nd
            pl = np.arange(Np, dtype=np.int64)
            Mn = np.zeros((Nd, Nd))
            for l in range(Nd):
                for n in range(Nd):
                    Mn[n, l] = (2 * l + 1) / 2 * Pl[n][l]
            Dn = np.linalg.inv(Mn)
        elif btype == "galerkin-d":
            Np = Nd
            pl = np.arange(Np, dtype=np.int64)
            Dn = np.zeros((Nd, Nd))
            for l in range(Nd):
                for n in range(Nd):
                    Dn[l, n] = w[n] * Pl[n][l]
            Mn = np.linalg.inv(Dn)
        else:
            raise ValueError("Unknown method.")
        return Np, Mn, Dn, pl, np.zeros(Np, dtype=np.int64)
    from .sphere import angular_polynomial_basis_sphere

    return angular_polynomial_basis_sphere(Om, w, L, btype, Qdims)


def surface_angular_polynomial_basis_face(Om, w, L: int, btype: str, Qdims: int, surface: str):
    """Half-range basis of one face (angular_polynomial_basis.jl:249-436):
    Np, Mn[Nd⁺,Np], Dn[Np,Nd⁺], n⁺_to_n, n_to_n⁺ (1-based, 0 = none), pl, pm."""
    surface = surface.upper()
    if Qdims == 1:
        mu = np.asarray(Om[0], dtype=float)
        if surface == "X-":
            idx = np.nonzero(mu > 0)[0]
            mup = mu[idx]
        elif surface == "X+":
            idx = np.nonzero(mu < 0)[0]
            mup = -mu[idx]
        else:
            raise ValueError("Unknown surface for 1D angular domain.")
        Ndp = len(idx)
        wp = np.asarray(w)[idx]
        Lb = max(L, galerkin_minimum_order(Ndp, 1)) if btype in ("galerkin-m", "galerkin-d") else L
        Pl = [half_range_legendre_polynomials_up_to_L(Lb, float(mup[k])) for k in range(Ndp)]
        Nd = len(mu)
        n_to_np = np.zeros(Nd, dtype=np.int64)
        for k, n in enumerate(idx):
            n_to_np[n] = k + 1
        if btype == "standard":
            Np = L + 1
            Mn = np.zeros((Ndp, Np)); Dn = np.zeros((Np, Ndp))
            for l in range(L + 1):
                for k in range(Ndp):
                    Mn[k, l] = Pl[k][l]
                    Dn[l, k] = wp[k] * Pl[k][l]
        elif btype == "galerkin-m":
            Np = Ndp
            Mn = np.zeros((Ndp, Ndp))
            for l in range(Ndp):
                for k in range(Ndp):
                    Mn[k, l] = Pl[k][l]
            Dn = np.linalg.inv(Mn)
        elif btype == "galerkin-d":
            Np = Ndp
            Dn = np.zeros((Ndp, Ndp))
            for l in range(Ndp):
                for k in range(Ndp):
                    Dn[l, k] = wp[k] * Pl[k][l]
            Mn = np.linalg.inv(Dn)
        else:
            raise ValueError("Unknown method.")
        pl = np.arange(Np, dtype=np.int64)
        return Np, Mn, Dn, idx + 1, n_to_np, pl, np.zeros(Np, dtype=np.int64)
    from .sphere import surface_basis_sphere_face

    return surface_basis_sphere_face(Om, w, L, btype, Qdims, surface)


def surface_angular_polynomial_basis(Om, w, L: int, btype: str, Qdims: int, Ndims: int):
    """All faces of a Cartesian geometry (angular_polynomial_basis.jl:208-247)."""
    faces = ["X-", "X+", "Y-", "Y+", "Z-", "Z+"][: 2 * Ndims]
    out = [surface_angular_polynomial_basis_face(Om, w, L, btype, Qdims, f) for f in faces]
    Np = out[-1][0]
    return (Np, [o[1] for o in out], [o[2] for o in out], [o[3] for o in out],
            [o[4] for o in out], [o[5] for o in out], [o[6] for o in out])


# --------------------------------------------------------------------------------------
# Closure weights (src/particle_transport/scheme_weights.jl:25-415)
# --------------------------------------------------------------------------------------


def axis_weights(scheme: str, order: int) -> np.ndarray:
    """ω of one axis, length order+1 (scheme_weights.jl:47-77). In the reference the
    multi-axis arrays ωx[:,m,t] repeat this vector for every other-axis index, so one
    vector per axis carries all of it."""
    M = order - 1
    w = np.zeros(M + 2)
    s = scheme.upper()
    if s == "DD" or (s == "AWD" and M == 0):
        w[0] = (-1) ** (M + 1)
        for n in range(M + 1):
            w[n + 1] = 1 - (-1) ** (M + 1 - n)
    elif s == "DG" or (s == "AWD" and M == 1):
        w[0] = 0.0
        w[1:] = 1.0
    elif s == "DG-":
        if M < 1:
            raise ValueError("DG- scheme require at least a 2nd-order p expansion.")
        w[0] = 0.0
        w[1:M + 1] = 1.0
        w[M + 1] = M / (2 * M + 1)
    elif s == "DG+":
        if M < 1:
            raise ValueError("DG+ scheme require at least a 2nd-order p expansion.")
        w[0] = 0.0
        w[1:M + 1] = 1.0
        w[M + 1] = 1001
    else:
        raise ValueError("Closure relation not implemented yet.")
    return w


def G6(j1: int, j2: int, j3: int) -> float:
    """𝒢₆: normalised triple-Legendre integral (src/tools/integrals.jl:254-276)."""
    def lf(n):
        return sum(math.log(k) for k in range(1, n + 1))

    Cjk = np.zeros((3, max(j1, j2, j3) // 2 + 1))
    for r, j in enumerate((j1, j2, j3)):
        for k in range(j // 2 + 1):
            Cjk[r, k] = (-1) ** k * math.exp(lf(2 * j - 2 * k) - lf(k) - lf(j - k) - lf(j - 2 * k))
    W = 0.0
    J = j1 + j2 + j3
    for k1 in range(j1 // 2 + 1):
        for k2 in range(j2 // 2 + 1):
            for k3 in range(j3 // 2 + 1):
                K = k1 + k2 + k3
                if (J - 2 * K) % 2 == 0:
                    W += Cjk[0, k1] * Cjk[1, k2] * Cjk[2, k3] * 1 / (J - 2 * K + 1)
    return W / 2 ** J


def scheme_weights(orders, schemes, Ndims: int, isCSD: bool):
    """Per-axis ω (x, y, z, E), 𝒞, is_adaptive, 𝒲 (scheme_weights.jl:25-415)."""
    for n in range(4):
        if orders[n] <= 0:
            raise ValueError("Scheme required at least a 1st-order polynomial expansion.")
    is_adaptive = any(s == "AWD" for s in schemes)
    if is_adaptive:
        schemes = ["AWD"] * 4
    w_axis = []
    for a in range(4):
        used = (a < Ndims) or (a == 3 and isCSD)
        w_axis.append(axis_weights(schemes[a], orders[a]) if used else axis_weights("DD", 1))
    nmax = max(orders)
    C = np.array([math.sqrt(2 * i - 1) for i in range(1, nmax + 1)])
    oE = orders[3]
    W = np.zeros((oE, oE, oE))
    for i in range(oE):
        for j in range(oE):
            for k in range(oE):
                W[i, j, k] = G6(i, j, k)
    return w_axis, C, is_adaptive, W


def get_schemes(scheme_type: dict, scheme_order: dict, axes, isCSD: bool, isFC: bool):
    """schemes, 𝒪, Nm (src/structures/SN.jl:520-544)."""
    schemes, O = [], []
    for x in ["x", "y", "z", "E"]:
        if x in axes or (isCSD and x == "E"):
            if x not in scheme_type:
                raise ValueError(f"Scheme type is not defined along {x}-axis.")
            if x not in scheme_order:
                raise ValueError(f"Scheme order is not defined along {x}-axis.")
            schemes.append(scheme_type[x].upper())
            O.append(int(scheme_order[x]))
        else:
            schemes.append("DD")
            O.append(1)
    if isFC:
        Nm = [O[1] * O[2] * O[3], O[0] * O[2] * O[3], O[0] * O[1] * O[3], O[0] * O[1] * O[2], int(np.prod(O))]
    else:
        Nm = [1 + (O[1] - 1) + (O[2] - 1) + (O[3] - 1), 1 + (O[0] - 1) + (O[2] - 1) + (O[3] - 1),
              1 + (O[0] - 1) + (O[1] - 1) + (O[3] - 1), 1 + (O[0] - 1) + (O[1] - 1) + (O[2] - 1),
              1 + sum(o - 1 for o in O)]
    return schemes, O, Nm


# --------------------------------------------------------------------------------------
# Angular Fokker-Planck matrix (fokker_planck_scattering_matrix.jl:29-48)
# --------------------------------------------------------------------------------------


def fokker_planck_galerkin(Nd: int, Mn: np.ndarray, Dn: np.ndarray, pl, Np: int):
    """Moment-preserving (Galerkin) ℳ and λ₀ (fokker_planck_galerkin.jl:25-52)."""
    Mp = np.diag([-float(l) * (l + 1) for l in pl[:Np]])
    Mn_ = Mn @ Mp @ Dn
    lam0 = 0.0
    for n in range(Nd):
        if Mn_[n, n] < -lam0:
            lam0 = -Mn_[n, n]
    for n in range(Nd):
        Mn_[n, n] += lam0
    return Dn @ Mn_ @ Mn, lam0


def fokker_planck_finite_difference_1d(N: int, qtype: str, Mn: np.ndarray, Dn: np.ndarray):
    """Finite-difference ℳ and λ₀, 1D branch (fokker_planck_finite_difference.jl:30-77)."""
    mu, w = quadrature(N, qtype, 1)
    index = np.argsort(mu, kind="stable")
    mun, wn = mu[index], w[index]
    b12 = np.zeros(N + 1)
    for n in range(2, N + 1):
        b12[n - 1] = b12[n - 2] - 2 * wn[n - 2] * mun[n - 2]
    Cm = np.zeros(N)
    for n in range(2, N + 1):
        Cm[n - 1] = b12[n - 1] / (wn[n - 1] * (mun[n - 1] - mun[n - 2]))
    Cp = np.zeros(N)
    for n in range(1, N):
        Cp[n - 1] = b12[n] / (wn[n - 1] * (mun[n] - mun[n - 1]))
    Cn = Cm + Cp
    lam0 = float(np.max(Cn))
    Mt = np.zeros((N, N))
    for n in range(N):
        Mt[n, n] = lam0 - Cn[n]
        if n >= 1:
            Mt[n, n - 1] = Cm[n]
        if n + 1 < N:
            Mt[n, n + 1] = Cp[n]
    Mnn = np.zeros((N, N))
    for n in range(N):
        for m in range(N):
            Mnn[index[n], index[m]] = Mt[n, m]
    return Dn @ Mnn @ Mn, lam0


def fokker_planck_finite_difference_glc(N: int, Qdims: int, Mn: np.ndarray, Dn: np.ndarray):
    """Finite-difference ℳ and λ₀ on the Gauss-Legendre-Chebychev product quadrature, the Qdims = 2
    and 3 branches of fokker_planck_finite_difference.jl:79-148 / 190-264 (Morel's polar
    differencing with β weights, azimuthal differencing scaled by γ_n; the azimuth spans [0, π]
    without wrap-around for Qdims = 2, [0, 2π] periodically for Qdims = 3), shifted by
    λ₀ = max |diag|, then Dn·ℳ·Mn."""
    mui, wi = gauss_legendre(N)
    idx = np.argsort(mui, kind="stable")
    mui, wi = mui[idx], wi[idx]
    Ni = len(mui)
    wj = math.pi / Ni
    na = Ni if Qdims == 2 else 2 * Ni          # azimuths per polar level
    om = np.array([math.pi * (n + 0.5) / Ni for n in range(na)])
    b12 = np.zeros(Ni + 1)
    d12 = np.zeros(Ni + 1)
    for n in range(1, Ni):
        b12[n] = b12[n - 1] - 2 * wi[n - 1] * mui[n - 1]
        d12[n] = (math.sqrt(1 - mui[n] ** 2) - math.sqrt(1 - mui[n - 1] ** 2)) / (mui[n] - mui[n - 1])
    gam = np.zeros(Ni)
    for n in range(Ni):
        cn = (b12[n + 1] * d12[n + 1] - b12[n] * d12[n]) / wi[n]
        Kn = 2 * (1 - mui[n] ** 2) + cn * math.sqrt(1 - mui[n] ** 2)
        gam[n] = (math.pi ** 2 * Kn) / (2 * Ni ** 2 * (1 - math.cos(math.pi / Ni)))
    M = np.zeros((Ni * na, Ni * na))

    def gap_left(i):   # ω_i − ω_(i−1) (wrapping through 2π in 3D)
        return om[i] - om[i - 1] if i > 0 else om[0] + 2 * math.pi - om[-1]

    def gap_right(i):  # ω_(i+1) − ω_i
        return om[i + 1] - om[i] if i < na - 1 else om[0] + 2 * math.pi - om[i]

    for n in range(Ni):
        a = 1.0 / (1 - mui[n] ** 2) * gam[n] / wj
        up = b12[n + 1] / (mui[n + 1] - mui[n]) if n < Ni - 1 else 0.0
        dn = b12[n] / (mui[n] - mui[n - 1]) if n > 0 else 0.0
        for i in range(na):
            ii = i + na * n
            # polar coupling
            M[ii, ii] -= (up + dn) / wi[n]
            if n > 0:
                M[ii, i + na * (n - 1)] += dn / wi[n]
            if n < Ni - 1:
                M[ii, i + na * (n + 1)] += up / wi[n]
            # azimuthal coupling
            if Qdims == 2:
                if i > 0:
                    M[ii, ii] -= a / gap_left(i)
                    M[ii, ii - 1] += a / gap_left(i)
                if i < na - 1:
                    M[ii, ii] -= a / gap_right(i)
                    M[ii, ii + 1] += a / gap_right(i)
            else:
                M[ii, ii] -= a / gap_left(i) + a / gap_right(i)
                M[ii, (i - 1) % na + na * n] += a / gap_left(i)
                M[ii, (i + 1) % na + na * n] += a / gap_right(i)
    lam0 = float(np.max(np.abs(np.diag(M))))
    M[np.diag_indices_from(M)] += lam0
    return Dn @ M @ Mn, lam0


def fokker_planck_differential_quadrature(N: int, qtype: str, Mn: np.ndarray, Dn: np.ndarray):
    """Differential-quadrature ℳ and λ₀, 1D (fokker_planck_differential_quadrature.jl:23-65):
    ℳ = (I − H²)·W¹² − 2·H·W¹ with the Lagrange first-derivative matrix W¹ on the nodes, shifted
    by λ₀ = max(−diag)."""
    mu, _ = quadrature(N, qtype, 1)
    mu = np.asarray(mu, dtype=float)
    H = np.diag(mu)
    I = np.eye(N)
    Pi = np.ones(N)
    for n in range(N):
        for m in range(N):
            if n != m:
                Pi[n] *= mu[n] - mu[m]
    W1 = np.zeros((N, N))
    for n in range(N):
        for m in range(N):
            if n != m:
                W1[n, m] = Pi[n] / ((mu[n] - mu[m]) * Pi[m])
    for n in range(N):
        for m in range(N):
            if n != m:
                W1[n, n] -= W1[n, m]
    M = (I - H @ H) @ (W1 @ W1) - 2 * H @ W1
    lam0 = 0.0
    for n in range(N):
        if M[n, n] < -lam0:
            lam0 = -M[n, n]
    M[np.diag_indices_from(M)] += lam0
    return Dn @ M @ Mn, lam0


def fokker_planck_scattering_matrix(N, Nd, qtype, Ndims, method, Mn, Dn, pl, Np, Qdims):
    """fokker_planck_scattering_matrix.jl:29-48."""
    if method == "finite-difference":
        if Qdims == 1:
            return fokker_planck_finite_difference_1d(N, qtype, Mn, Dn)
        if qtype == "gauss-legendre-chebychev":
            return fokker_planck_finite_difference_glc(N, Qdims, Mn, Dn)
        raise NotImplementedError("finite-difference Fokker-Planck on a non-product quadrature needs the "
                                  "spherical Voronoi weights, which are not built; use gauss-legendre-chebychev "
                                  "or the galerkin method")
    if method == "galerkin":
        return fokker_planck_galerkin(Nd, Mn, Dn, pl, Np)
    if method == "differential-quadrature":
        if Qdims != 1:
            raise ValueError("Differential quadrature unavailable in multidimensional geometry.")
        return fokker_planck_differential_quadrature(N, qtype, Mn, Dn)
    raise ValueError("Unknown method to treat the Fokker-Planck term.")
