"""The rearranged stencil sums of the substep kernels, checked in float64
against the node-by-node sums of the reference's P2G / G2P loops
(simulation.py:137-271, 304-383).

The kernels form per-node factors from per-axis ones and accumulate moments
that are finished after the 27-node loop:
  * APIC payload  m (v + C dpos) = K + Cd o,  Cd = m dx C,  K = m v - Cd fx,
    dpos = (o - fx) dx, o the node's offsets (0, 1, 2) per axis;
  * sum W g (x) dpos = dx (sum W g (x) o - (sum W g) (x) fx);
  * APIC gather C = 4/dx sum W g (x) (o - fx) = 4/dx (mo - v fx^T);
  * sum (g . P3) (H d3)_b = sum_c (sum (g . P3) H_bc) d3_c.
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
