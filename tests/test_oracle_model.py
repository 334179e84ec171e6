"""The FP64 modelling/adjoint oracle (oracle/oracle_model.c) checked against itself: the
forward/adjoint pair passes the dot-product test and the gradient matches central finite
differences of the misfit. (The reference has no adjoint, so nothing else can pin it.)"""
import numpy as np
import pytest

from hpcscan_b200 import layout as L
from hpcscan_b200.modeling import ricker, sponge_table, stable_dt

ORDER, DX, NT = 8, 10.0, 70


def problem(seed=0, n=(22, 18, 20)):
    lay = L.b200_layout(3, *n, order=ORDER, prec="f64")
    rng = np.random.default_rng(seed)
    v = np.zeros((lay.n3, lay.n2, lay.n1))
    sl = (slice(lay.a3.inner_start, lay.a3.inner_end + 1), slice(lay.a2.inner_start, lay.a2.inner_end + 1),
          slice(lay.a1.inner_start, lay.a1.inner_end + 1))
    v[sl] = 2000.0 + 300.0 * rng.standard_normal(v[sl].shape).clip(-2, 2)
    dt = stable_dt(ORDER, DX, 2600.0)
    m = np.zeros_like(v)
    m[sl] = 1.0 / v[sl] ** 2
    g = [sponge_table(ax.n, ax.inner_start, ax.inner_end, 4).astype(np.float64)
         for ax in (lay.a1, lay.a2, lay.a3)]
    G = (g[2][:, None, None] * g[1][None, :, None] * g[0][None, None, :]).reshape(-1)
    def flat(i1, i2, i3):
        return (lay.a1.inner_start + i1) + (lay.a2.inner_start + i2) * lay.n1 + \
            (lay.a3.inner_start + i3) * lay.n1 * lay.n2
    src = flat(4, 9, 10)
    rec = np.array([flat(2, j, k) for j in range(1, n[1] - 1, 3) for k in range(1, n[2] - 1, 3)])
    inv2 = (1.0 / DX ** 2,) * 3
    wav = ricker(40.0, dt, NT).astype(np.float64)
    return lay, m.reshape(-1), sl, G, src, rec, inv2, wav, dt


def coef(m, dt):
    c = np.zeros_like(m)
    nz = m > 0
    c[nz] = dt * dt / m[nz]
    return c


def test_dot_product_forward_adjoint():
    from oracle import oracle
    lay, m, sl, G, src, rec, inv2, wav, dt = problem()
    C = coef(m, dt)
    amp = 3.0
    d = oracle.model_forward(lay, C, G, src, amp, wav, rec, inv2)
    r = np.random.default_rng(5).standard_normal(d.shape)
    w_src = oracle.model_adjoint(lay, C, G, r, rec, src, inv2)
    lhs = float((d * r).sum())
    rhs = float((amp * wav * w_src).sum() / C[src])
    assert lhs == pytest.approx(rhs, rel=1e-11), (lhs, rhs)


def test_gradient_matches_central_differences():
    from oracle import oracle
    lay, m, sl, G, src, rec, inv2, wav, dt = problem(seed=1)
    mtrue = m.copy().reshape(lay.n3, lay.n2, lay.n1)
    mtrue[sl] *= 1.0 + 0.05 * np.random.default_rng(2).standard_normal(mtrue[sl].shape).clip(-2, 2)
    dobs = oracle.model_forward(lay, coef(mtrue.reshape(-1), dt), G, src, 1.0, wav, rec, inv2)
    J, g = oracle.model_gradient(lay, coef(m, dt), G, src, 1.0, wav, rec, inv2, dobs, dt)
    dm = np.zeros_like(m).reshape(lay.n3, lay.n2, lay.n1)
    dm[sl] = np.random.default_rng(3).standard_normal(dm[sl].shape)
    dm = dm.reshape(-1) * 1e-2 * np.abs(m).max()
    eps = 1e-3
    Jp = 0.5 * ((oracle.model_forward(lay, coef(m + eps * dm, dt), G, src, 1.0, wav, rec, inv2) - dobs) ** 2).sum()
    Jm = 0.5 * ((oracle.model_forward(lay, coef(m - eps * dm, dt), G, src, 1.0, wav, rec, inv2) - dobs) ** 2).sum()
    fd = (Jp - Jm) / (2 * eps)
    an = float((g * dm).sum())
    assert J > 0 and an != 0.0
    assert fd == pytest.approx(an, rel=1e-5), (fd, an)
