"""The analytic solution of Underworld's Velic solCx benchmark, for the convergence test.

Problem (Underworld/SysTest/AnalyticPlugins/Velic_solCx/solCx_main.tex, testVelicSolCx.xml):
Stokes flow in the unit square with free-slip walls, viscosity η_A for x < x_c and η_B for
x > x_c, body force f = (0, F0 sin(k_z y) cos(k_x x)) with k_z = n_z π, k_x = n_x π.

Derived here from the stream-function form (not taken from the reference's generated
solCx.cxx): u = ∂ψ/∂y, v = −∂ψ/∂x, ψ = Φ(x) sin(k_z y) meets the free-slip conditions at
y = 0, 1.  In each region η(Φ'''' − 2k_z²Φ'' + k_z⁴Φ) = −F0 k_x sin(k_x x), so
Φ = (a + bx) cosh(k_z x) + (c + dx) sinh(k_z x) + A sin(k_x x),
A = −F0 k_x / (η (k_x² + k_z²)²).  The eight constants follow from free slip at x = 0, 1
(Φ = Φ'' = 0) and, at x = x_c, continuity of u, v (Φ, Φ') and of the tractions
σ_xy (η(Φ'' + k_z²Φ)) and σ_xx (η(Φ''' − 3k_z²Φ')).  The pressure is
p = P(x) cos(k_z y), P = (η(Φ''' − k_z²Φ') − F0 cos(k_x x)) / k_z, whose mean over the box
is zero."""
import numpy as np


def _region_coeffs(eta_a, eta_b, xc, kz, kx, F0):
    A = np.array([-F0 * kx / (eta * (kx * kx + kz * kz) ** 2) for eta in (eta_a, eta_b)])

    def basis(x, m):
        ch, sh = np.cosh(kz * x), np.sinh(kz * x)
        gc = lambda j: kz ** j * (ch if j % 2 == 0 else sh)  # noqa: E731  (cosh)^(j)
        gs = lambda j: kz ** j * (sh if j % 2 == 0 else ch)  # noqa: E731  (sinh)^(j)
        xgc = x * gc(m) + (m * gc(m - 1) if m > 0 else 0.0)
        xgs = x * gs(m) + (m * gs(m - 1) if m > 0 else 0.0)
        return np.array([gc(m), xgc, gs(m), xgs])

    def part(R, x, m):
        s = (np.sin(kx * x), np.cos(kx * x), -np.sin(kx * x), -np.cos(kx * x))[m % 4]
        return A[R] * kx ** m * s

    eta = (eta_a, eta_b)
    M, rhs = np.zeros((8, 8)), np.zeros(8)
    r = 0
    for R, x0 in ((0, 0.0), (1, 1.0)):
        for m in (0, 2):
            M[r, 4 * R:4 * R + 4] = basis(x0, m)
            rhs[r] = -part(R, x0, m)
            r += 1
    for m in (0, 1):
        M[r, :4], M[r, 4:] = basis(xc, m), -basis(xc, m)
        rhs[r] = part(1, xc, m) - part(0, xc, m)
        r += 1
    for combo in ((2, 0, kz * kz), (3, 1, -3.0 * kz * kz)):
        hi, lo, w = combo
        for R, sgn in ((0, 1.0), (1, -1.0)):
            M[r, 4 * R:4 * R + 4] = sgn * eta[R] * (basis(xc, hi) + w * basis(xc, lo))
            rhs[r] -= sgn * eta[R] * (part(R, xc, hi) + w * part(R, xc, lo))
        r += 1
    return np.linalg.solve(M, rhs), A


def solcx(x, y, eta_a=100.0, eta_b=1.0, xc=0.5, nz=2, nx=1, F0=1.0):
    """u, v, p and the strain rate (ε_xx, ε_yy, ε_xy) at the points (x, y)."""
    kz, kx = nz * np.pi, nx * np.pi
    c, A = _region_coeffs(eta_a, eta_b, xc, kz, kx, F0)
    x, y = np.asarray(x, float), np.asarray(y, float)
    R = (x >= xc).astype(int)
    cR = c.reshape(2, 4)[R]  # [npts, 4]
    ch, sh = np.cosh(kz * x), np.sinh(kz * x)
    phi = []
    for m in range(4):
        gc = kz ** m * (ch if m % 2 == 0 else sh)
        gs = kz ** m * (sh if m % 2 == 0 else ch)
        gc1 = kz ** (m - 1) * (sh if m % 2 == 0 else ch) if m > 0 else 0.0
        gs1 = kz ** (m - 1) * (ch if m % 2 == 0 else sh) if m > 0 else 0.0
        hom = cR[:, 0] * gc + cR[:, 1] * (x * gc + m * gc1) + cR[:, 2] * gs + cR[:, 3] * (x * gs + m * gs1)
        s = (np.sin(kx * x), np.cos(kx * x), -np.sin(kx * x), -np.cos(kx * x))[m]
        phi.append(hom + A[R] * kx ** m * s)
    eta = np.where(R == 0, eta_a, eta_b)
    cz, sz = np.cos(kz * y), np.sin(kz * y)
    u = phi[0] * kz * cz
    v = -phi[1] * sz
    p = (eta * (phi[3] - kz * kz * phi[1]) - F0 * np.cos(kx * x)) / kz * cz
    exx = phi[1] * kz * cz
    eyy = -phi[1] * kz * cz
    exy = 0.5 * (-phi[0] * kz * kz - phi[2]) * sz
    return u, v, p, np.stack([exx, eyy, exy], axis=-1)


def relative_errors(n, u_nodal, p_elem, **kw):
    """The relative L2 errors sqrt(Σ (num − ana)² w detJ / Σ ana² w detJ) of vx, vy, p and
    the strain-rate components on the n × n unit-square Q1-P0 mesh, integrated with 2 × 2
    Gauss points per element (FieldTest over the deck's gaussSwarm); both pressures taken
    with zero mean over the box.  u_nodal is component-major [2, (n+1)²]."""
    h = 1.0 / n
    g = np.array([-1.0, 1.0]) / np.sqrt(3.0)
    I, J = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
    I, J = I.ravel(), J.ravel()
    ux = u_nodal[0].reshape(n + 1, n + 1)  # [j, i]
    uy = u_nodal[1].reshape(n + 1, n + 1)
    pm = p_elem - p_elem.mean()
    num, den = np.zeros(6), np.zeros(6)
    for gx in g:
        for gy in g:
            sx, sy = 0.5 * (1 + gx), 0.5 * (1 + gy)
            X, Y = (I + sx) * h, (J + sy) * h
            N = [(1 - sx) * (1 - sy), sx * (1 - sy), (1 - sx) * sy, sx * sy]
            dNx = np.array([-(1 - sy), (1 - sy), -sy, sy]) / h
            dNy = np.array([-(1 - sx), -sx, (1 - sx), sx]) / h
            corners = [(J, I), (J, I + 1), (J + 1, I), (J + 1, I + 1)]
            vx = sum(N[a] * ux[corners[a]] for a in range(4))
            vy = sum(N[a] * uy[corners[a]] for a in range(4))
            dux = sum(dNx[a] * ux[corners[a]] for a in range(4))
            duy = sum(dNy[a] * ux[corners[a]] for a in range(4))
            dvx = sum(dNx[a] * uy[corners[a]] for a in range(4))
            dvy = sum(dNy[a] * uy[corners[a]] for a in range(4))
            au, av, ap, ae = solcx(X, Y, **kw)
            numeric = [vx, vy, pm, dux, dvy, 0.5 * (duy + dvx)]
            exact = [au, av, ap, ae[:, 0], ae[:, 1], ae[:, 2]]
            w = h * h / 4.0
            for c in range(6):
                num[c] += np.sum((numeric[c] - exact[c]) ** 2) * w
                den[c] += np.sum(exact[c] ** 2) * w
    return np.sqrt(num / den)
