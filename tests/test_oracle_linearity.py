"""The premise of the shared stage transforms, checked on the oracle's
restatement of the reference projection (CPU): a fast stage projects
(u, v, w + sdt b) with b the half-level buoyancy of the anchor theta', and
that projection -- divergence, compatibility, the Thomas solves with the zero
mode, the gradient correction -- is linear, so every stage's result and
potential equal P(u, v, w) + sdt P(0, 0, b).  The B200 step forms each stage's
divergence spectrum from one x transform of (u, v, w) and one of b on that
basis (integrator.py:398-505 for the stages, tendency.py:717-790 and
poisson.py:98-383 for the projection)."""
import numpy as np

from oracle import lh82 as O


def _state(rng, nx, ny, nz, Lx, Ly):
    x = (np.arange(nx) + 0.5) / nx * 2 * np.pi
    y = (np.arange(ny) + 0.5) / ny * 2 * np.pi
    X, Y = np.meshgrid(x, y, indexing="ij")
    zf = np.linspace(0.1, 0.9, nz)
    zh = np.linspace(0.0, 1.0, nz + 1)
    u = 20 * np.sin(X)[:, :, None] * np.cos(Y)[:, :, None] * (1 - zf)[None, None, :]
    v = -15 * np.cos(2 * X)[:, :, None] * np.sin(Y)[:, :, None] * zf[None, None, :]
    w = 0.5 * np.sin(X + Y)[:, :, None] * np.sin(np.pi * zh)[None, None, :]
    th = 2.0 * np.exp(-((X - np.pi) ** 2 + (Y - np.pi) ** 2))[:, :, None] * np.sin(np.pi * zf)
    u = u + 1e-3 * rng.standard_normal(u.shape)
    v = v + 1e-3 * rng.standard_normal(v.shape)
    return u, v, w, th


def _project(u, v, w, nx, ny, nz, Lx, Ly, Lz, rho0):
    st = O.State(u.copy(), v.copy(), w.copy(), np.zeros_like(u), np.zeros_like(u), 0.0)
    O.Projection(nx, ny, nz, Lx, Ly, Lz).apply(st, rho0)
    return st


def test_stage_projection_is_linear_in_the_stage_increment():
    nx, ny, nz = 32, 24, 16
    Lx, Ly, Lz = nx * 10e3, ny * 10e3, 16e3
    _, rho0, th0 = O.build_base_state(nz, Lz)
    rng = np.random.default_rng(5)
    u, v, w, th = _state(rng, nx, ny, nz, Lx, Ly)
    b = O.buoyancy_half(th, th0)
    a = _project(u, v, w, nx, ny, nz, Lx, Ly, Lz, rho0)
    z = np.zeros_like(u)
    pb = _project(z, z, b, nx, ny, nz, Lx, Ly, Lz, rho0)
    dt = 60.0
    for alpha in (1.0 / 3.0, 0.5, 1.0):
        sdt = alpha * dt
        s = _project(u, v, w + sdt * b, nx, ny, nz, Lx, Ly, Lz, rho0)
        for f in ("u", "v", "w", "projection_potential"):
            ref = getattr(s, f)
            lin = getattr(a, f) + sdt * getattr(pb, f)
            err = np.max(np.abs(lin - ref)) / np.max(np.abs(ref))
            assert err <= 1e-12, (alpha, f, err)
    # the divergence the stage's solve starts from, in spectral form
    s0 = O.Poisson(nx, ny, nz, Lx, Ly, Lz)
    rf, rh = rho0, O.rho_half_levels(rho0)
    dz = Lz / nz
    d_a = O.anelastic_divergence(u, v, w, rf, rh, s0.kx, s0.ky, dz)
    d_b = O.anelastic_divergence(z, z, b, rf, rh, s0.kx, s0.ky, dz)
    d_s = O.anelastic_divergence(u, v, w + dt * b, rf, rh, s0.kx, s0.ky, dz)
    assert np.max(np.abs(d_a + dt * d_b - d_s)) <= 1e-12 * np.max(np.abs(d_s))
