"""Oracle for the NS time-stepper operators of the reference (test and CPU-baseline infrastructure only).

Restates ``Anisotropic Resistivity Tomography/scripts/naiver_stokes_3D.py`` (and the same
functions of ``Urban Modelling/AI_HFM_v3.ipynb`` cell 19) in NumPy.  Arrays are (Z, Y, X);
the reference's (1, nx, ny, nz, 1) tensors with indices [0, z, y, x, 0] (its boundary
functions address axis 3 as x: inflow at index 0, outflow at nx-1).
"""
import numpy as np

from . import tfops


def bc_velocity(u, v, w, ub):
    """``boundary_condition_velocity`` (naiver_stokes_3D.py:420-447): plane assignments in
    the reference's order; every copied plane is read from the *input* arrays (the reference
    copies ``tf.Variable(values_u)`` before assigning)."""
    u0, v0, w0 = u, v, w
    u, v, w = u.copy(), v.copy(), w.copy()
    u[:, :, 0] = ub
    v[:, :, 0] = 0
    w[:, :, 0] = 0
    u[:, :, -1] = ub
    v[:, :, -1] = 0
    w[:, :, -1] = 0
    u[:, 0, :] = u0[:, 1, :]
    v[:, 0, :] = 0
    w[:, 0, :] = 0
    u[:, -1, :] = u0[:, -2, :]
    v[:, -1, :] = 0
    w[:, -1, :] = 0
    u[0, :, :] = 0
    v[0, :, :] = 0
    w[0, :, :] = 0
    u[-1, :, :] = u0[-2, :, :]
    v[-1, :, :] = v0[-2, :, :]
    w[-1, :, :] = 0
    return u, v, w


def bc_pressure(p):
    """``boundary_condition_pressure`` (naiver_stokes_3D.py:452-462)."""
    p0 = p
    p = p.copy()
    p[:, :, -1] = 0
    p[:, :, 0] = p0[:, :, 1]
    p[:, 0, :] = p0[:, 1, :]
    p[:, -1, :] = p0[:, -2, :]
    p[0, :, :] = p0[1, :, :]
    p[-1, :, :] = p0[-2, :, :]
    return p


def bc_source(b):
    """``boundary_condition_source`` (naiver_stokes_3D.py:467-473)."""
    b = b.copy()
    b[:, :, 0] = b[:, :, 1]
    return b


def bluff_body(u, v, w, sigma, dt):
    """``bluff_body`` (naiver_stokes_3D.py:478-483): u / (1 + dt sigma)."""
    d = (1.0 + dt * sigma).astype(u.dtype)
    return u / d, v / d, w / d


def momentum_rhs(phi, au, av, aw, Kdif, Kx, Ky, Kz, dt=np.float32):
    """a = Dif(phi) - u Dx(phi) - v Dy(phi) - w Dz(phi) (naiver_stokes_3D.py:580-592)."""
    c = lambda K: tfops.conv3d_same(phi, K, dt)
    return c(Kdif) - au * c(Kx) - av * c(Ky) - aw * c(Kz)


def momentum(u, v, w, ub, Kdif, Kx, Ky, Kz):
    """Two-stage momentum update of naiver_stokes_3D.py:580-622: b = u + a(u)/2, BC(b),
    u += a(b) with the stage-2 advecting velocity b."""
    bu = 0.5 * momentum_rhs(u, u, v, w, Kdif, Kx, Ky, Kz) + u
    bv = 0.5 * momentum_rhs(v, u, v, w, Kdif, Kx, Ky, Kz) + v
    bw = 0.5 * momentum_rhs(w, u, v, w, Kdif, Kx, Ky, Kz) + w
    bu, bv, bw = bc_velocity(bu, bv, bw, ub)
    u1 = u + momentum_rhs(bu, bu, bv, bw, Kdif, Kx, Ky, Kz)
    v1 = v + momentum_rhs(bv, bu, bv, bw, Kdif, Kx, Ky, Kz)
    w1 = w + momentum_rhs(bw, bu, bv, bw, Kdif, Kx, Ky, Kz)
    return u1, v1, w1


def pressure_gradient(p, u, v, w, Kx, Ky, Kz):
    """u -= pu(p), v -= pv(p), w -= pw(p) (naiver_stokes_3D.py:631-633)."""
    return (u - tfops.conv3d_same(p, Kx), v - tfops.conv3d_same(p, Ky),
            w - tfops.conv3d_same(p, Kz))


def divergence_rhs(u, v, w, Su, Sv, Sw):
    """b = -(Su(u) + Sv(v) + Sw(w)), then boundary_condition_source (naiver_stokes_3D.py:641-642)."""
    b = -(tfops.conv3d_same(u, Su) + tfops.conv3d_same(v, Sv) + tfops.conv3d_same(w, Sw))
    return bc_source(b)


def step(u, v, w, p, sigma, dt, ub, Kdif, Kx, Ky, Kz, Su, Sv, Sw, Kp, n_levels, multi_itr,
         pressure=None):
    """One reference time step (naiver_stokes_3D.py:571-727) with the reference's pressure
    multigrid (sawtooth NS form, ``multi_itr`` cycles), or with ``pressure(p, b) -> p``
    solving the pressure equation instead when it is given."""
    from . import mg
    u, v, w = bc_velocity(u, v, w, ub)
    p = bc_pressure(p)
    u, v, w = momentum(u, v, w, ub, Kdif, Kx, Ky, Kz)
    u, v, w = bluff_body(u, v, w, sigma, dt)
    u, v, w = pressure_gradient(p, u, v, w, Kx, Ky, Kz)
    u, v, w = bc_velocity(u, v, w, ub)
    b = divergence_rhs(u, v, w, Su, Sv, Sw)
    if pressure is not None:
        p = pressure(p, b)
    else:
        ops = mg.hierarchy(mg.Stencil27(Kp), n_levels)
        for _ in range(multi_itr):
            p = mg.sawtooth_cycle(ops, p, b, fine_smooth=False, zero_xend=True)
    p = bc_pressure(p)
    u, v, w = pressure_gradient(p, u, v, w, Kx, Ky, Kz)
    u, v, w = bc_velocity(u, v, w, ub)
    u, v, w = bluff_body(u, v, w, sigma, dt)
    return u, v, w, p


def pg_dissipation(u, v, w, sigma, dt, eps_k, Kdif, Kx, Ky, Kz):
    """``Petrov_Galerkin_dissipation`` (``Urban Modelling/INHALE_demo.ipynb`` cell 20), float32
    in the cell's order: velocities damped by (1 + dt sigma), coefficients k_f clipped at 0.5,
    then 1.5 (k_f D(f) + D(f k_f) - f D(k_f)) with D the diffusion stencil."""
    f32 = np.float32
    c = lambda a, K: tfops.conv3d_same(a, K)
    den = (f32(1) + f32(dt) * np.asarray(sigma, f32)).astype(f32)
    u, v, w = (np.asarray(a, f32) / den for a in (u, v, w))
    speed = (np.abs(u) + np.abs(v)) + np.abs(w)
    out = []
    for f in (u, v, w):
        k = f32(2) * np.abs(speed / f32(3) * c(f, Kdif)) / (
            f32(eps_k) + ((np.abs(c(f, Kx)) + np.abs(c(f, Ky))) + np.abs(c(f, Kz))) / f32(3))
        k = np.minimum(k, f32(0.5)) / den
        out.append(f32(1.5) * ((k * c(f, Kdif) + c(f * k, Kdif)) - f * c(k, Kdif)))
    return out


def momentum_pg(u, v, w, ub, sigma, dt, eps_k, Kdif, Kx, Ky, Kz):
    """The two-stage momentum update of ``INHALE_demo.ipynb`` cell 24 with Petrov-Galerkin
    dissipation in place of the diffusion stencil: a = k - u Dx - v Dy - w Dz (stage 1 on u^n,
    b = u + a / 2, BC(b); stage 2 with k and the advecting velocity from b, u += a(b))."""
    c = lambda a, K: tfops.conv3d_same(a, K)
    k = pg_dissipation(u, v, w, sigma, dt, eps_k, Kdif, Kx, Ky, Kz)
    b = [(0.5 * (((kf - u * c(f, Kx)) - v * c(f, Ky)) - w * c(f, Kz)) + f)
         for kf, f in zip(k, (u, v, w))]
    bu, bv, bw = bc_velocity(*b, ub)
    kb = pg_dissipation(bu, bv, bw, sigma, dt, eps_k, Kdif, Kx, Ky, Kz)
    return tuple(f + (((kf - bu * c(g, Kx)) - bv * c(g, Ky)) - bw * c(g, Kz))
                 for kf, f, g in zip(kb, (u, v, w), (bu, bv, bw)))
