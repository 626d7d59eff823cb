"""The rearranged stencil sums of the substep kernels, checked in float64
against the node-by-node sums of the reference's P2G / G2P loops
(simulation.py:137-271, 304-383).

The kernels form per-node factors from per-axis ones and accumulate moments
that are finished after the 27-node loop:
  * APIC payload  m (v + C dpos) = K + Cd o,  Cd = m dx C,  K = m v - Cd fx,
    dpos = (o - fx) dx, o the node's offsets (0, 1, 2) per axis;
  * sum W g (x) dpos = dx (sum W g (x) o - (sum W g) (x) fx);
  * APIC gather C = 4/dx sum W g (x) (o - fx) = 4/dx (mo - v fx^T);
  * sum (g . P3) (H d3)_b = sum_c (sum (g . P3) H_bc) d3_c;
  * sum factorisation: sums over the stencil's z column first, per (x, y)
    column, scaled by the column's x and y factors afterwards.
"""
import numpy as np


def bspline(fx):
    a, b, c = 1.5 - fx, fx - 1.0, fx - 0.5
    return np.array([0.5 * a * a, 0.75 - b * b, 0.5 * c * c]), np.array([fx - 1.5, 2 * (1 - fx), fx - 0.5])


DD = np.array([1.0, -2.0, 1.0])


def _case(seed):
    rng = np.random.default_rng(seed)
    fx = rng.uniform(0.5, 1.5, 3)
    ws, dws = zip(*(bspline(f) for f in fx))
    return (rng, fx, np.array(ws), np.array(dws), 1.0 / 64, rng.uniform(0.1, 1.0), rng.normal(size=(3, 3)),
            rng.normal(size=3), rng.normal(size=(3, 3, 3, 4)))


def _nodes():
    for oi in range(3):
        for oj in range(3):
            for ok in range(3):
                yield oi, oj, ok


def test_separable_payload_and_momentum_moments():
    for seed in range(8):
        rng, fx, w, dw, dx, m, C, v, g = _case(seed)
        Cd = m * dx * C
        K = m * v - Cd @ fx
        sp = np.zeros(3); spd = np.zeros((3, 3)); mo = np.zeros((3, 3)); pay_err = 0.0
        for o in _nodes():
            W = w[0][o[0]] * w[1][o[1]] * w[2][o[2]]
            dpos = (np.array(o) - fx) * dx
            pay = m * (v + C @ dpos)
            pay_err = max(pay_err, np.abs(pay - (K + Cd @ np.array(o))).max())
            bp = g[o][:3]
            sp += W * bp
            spd += W * np.outer(bp, dpos)
            mo += W * np.outer(bp, o)
        assert pay_err < 1e-12
        np.testing.assert_allclose(dx * (mo - np.outer(sp, fx)), spd, rtol=1e-10, atol=1e-14)


def test_apic_gather_from_moments():
    for seed in range(8):
        rng, fx, w, dw, dx, m, C, v, g = _case(seed)
        inv_dx = 1.0 / dx
        vsum = np.zeros(3); Cref = np.zeros((3, 3)); mo = np.zeros((3, 3))
        for o in _nodes():
            W = w[0][o[0]] * w[1][o[1]] * w[2][o[2]]
            ga = g[o][:3]
            vsum += W * ga
            Cref += 4 * W * inv_dx * np.outer(ga, np.array(o) - fx)
            mo += W * np.outer(ga, o)
        np.testing.assert_allclose(4 * inv_dx * (mo - np.outer(vsum, fx)), Cref, rtol=1e-10, atol=1e-12)


def test_hessian_term_from_symmetric_moments():
    for seed in range(8):
        rng, fx, w, dw, dx, m, C, v, g = _case(seed)
        inv_dx = 1.0 / dx
        P3, d3 = rng.normal(size=3), rng.normal(size=3)
        ref = np.zeros(3); hs = np.zeros((3, 3))
        for o in _nodes():
            i, j, k = o
            f = [(w[0][i], dw[0][i], DD[i]), (w[1][j], dw[1][j], DD[j]), (w[2][k], dw[2][k], DD[k])]
            H = np.empty((3, 3))
            for b in range(3):
                for c in range(3):
                    prod = 1.0
                    for a in range(3):
                        if a == b == c:
                            prod *= f[a][2]
                        elif a == b or a == c:
                            prod *= f[a][1]
                        else:
                            prod *= f[a][0]
                    H[b, c] = prod * inv_dx * inv_dx
            sP = g[o][:3] @ P3
            ref += sP * (H @ d3)
            hs += sP * H
        np.testing.assert_allclose(hs @ d3, ref, rtol=1e-10, atol=1e-9)
        np.testing.assert_allclose(hs, hs.T, rtol=1e-12, atol=1e-9)


def test_sum_factorised_triangle_adjoint_sums():
    """The per-column sums of k_tri_adj's stencil loop (Rw, Rk, Re, Tw, Te,
    Td, Sw, Se over the z nodes of each (x, y) column) give the node-by-node
    sums of the APIC moments, the normal force's adjoint terms and the
    position adjoint."""
    for seed in range(8):
        rng, fx, w, dw, dx, m, C, v, g = _case(seed)
        inv_dx = 1.0 / dx
        ed = dw * inv_dx
        ddc = DD * inv_dx * inv_dx
        P3, d3 = rng.normal(size=3), rng.normal(size=3)
        Cm = m * dx * C
        K = m * v - Cm @ fx
        # node by node
        sp = np.zeros(3); mo = np.zeros((3, 3)); g3 = np.zeros(3); sg = np.zeros(3); bx = np.zeros(3); hs = np.zeros(6)
        for (i, j, k) in _nodes():
            W = w[0][i] * w[1][j] * w[2][k]
            gW = np.array([ed[0][i] * w[1][j] * w[2][k], w[0][i] * ed[1][j] * w[2][k], w[0][i] * w[1][j] * ed[2][k]])
            H = np.array([ddc[i] * w[1][j] * w[2][k], ed[0][i] * ed[1][j] * w[2][k], ed[0][i] * w[1][j] * ed[2][k],
                          w[0][i] * ddc[j] * w[2][k], w[0][i] * ed[1][j] * ed[2][k], w[0][i] * w[1][j] * ddc[k]])
            bp, gw = g[i, j, k][:3], g[i, j, k][3]
            sP = bp @ P3
            s_n = gw * m + bp @ (K + Cm @ np.array([i, j, k]))
            sp += W * bp
            mo += W * np.outer(bp, [i, j, k])
            g3 += (gW @ d3) * bp
            sg += sP * gW
            bx += s_n * gW
            hs += sP * H
        # factorised as in the kernel
        fsp = np.zeros(3); fmo = np.zeros((3, 3)); fg3 = np.zeros(3); fsg = np.zeros(3); fbx = np.zeros(3)
        fhs = np.zeros(6)
        for i in range(3):
            for j in range(3):
                w01, e0w1, w0e1 = w[0][i] * w[1][j], ed[0][i] * w[1][j], w[0][i] * ed[1][j]
                e0e1, d0w1, w0d1 = ed[0][i] * ed[1][j], ddc[i] * w[1][j], w[0][i] * ddc[j]
                Rw = np.zeros(3); Rk = np.zeros(3); Re = np.zeros(3)
                Tw = Te = Td = Sw = Se = 0.0
                for k in range(3):
                    bp, gw = g[i, j, k][:3], g[i, j, k][3]
                    sP = bp @ P3
                    s_n = gw * m + bp @ (K + Cm @ np.array([i, j, k]))
                    Rw += w[2][k] * bp
                    Rk += k * w[2][k] * bp
                    Re += ed[2][k] * bp
                    Tw += w[2][k] * sP
                    Te += ed[2][k] * sP
                    Td += ddc[k] * sP
                    Sw += w[2][k] * s_n
                    Se += ed[2][k] * s_n
                fsp += w01 * Rw
                fmo += np.outer(w01 * Rw, [i, j, 0]) + np.outer(w01 * Rk, [0, 0, 1])
                fg3 += (d3[0] * e0w1 + d3[1] * w0e1) * Rw + d3[2] * w01 * Re
                fsg += np.array([e0w1 * Tw, w0e1 * Tw, w01 * Te])
                fhs += np.array([d0w1 * Tw, e0e1 * Tw, e0w1 * Te, w0d1 * Tw, w0e1 * Te, w01 * Td])
                fbx += np.array([e0w1 * Sw, w0e1 * Sw, w01 * Se])
        for a, b in ((sp, fsp), (mo, fmo), (g3, fg3), (sg, fsg), (bx, fbx), (hs, fhs)):
            np.testing.assert_allclose(b, a, rtol=1e-10, atol=1e-9 * max(1.0, np.abs(a).max()))
