"""Known answers from mathematics, on the CPU oracle: e^{iQ} against a
general matrix exponential, the order of Luscher's RK3 integrator, and the
flow's monotone plaquette."""
import numpy as np
import pytest
from scipy.linalg import expm


def random_hermitian_traceless(n, scale, rng):
    a = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
    h = (a + np.conj(np.swapaxes(a, -1, -2))) / 2
    h -= np.eye(3) * np.trace(h, axis1=-2, axis2=-1)[:, None, None] / 3
    return h * scale


def to_real(c):
    return np.stack([c.real, c.imag], axis=-1).reshape(c.shape[0], 18)


def to_complex(r):
    a = r.reshape(-1, 3, 3, 2)
    return a[..., 0] + 1j * a[..., 1]


@pytest.mark.parametrize("scale", [1e-3, 0.1, 1.0, 4.0])
def test_oracle_exponential_against_expm(oracle, scale):
    rng = np.random.default_rng(int(scale * 1000) + 1)
    q = random_hermitian_traceless(64, scale, rng)
    got = to_complex(oracle.su3_exp(to_real(q)))
    want = np.array([expm(1j * m) for m in q])
    assert np.abs(got - want).max() < 1e-13 * max(1.0, scale ** 2)
    assert np.abs(np.linalg.det(got) - 1).max() < 1e-13
    assert np.abs(got @ np.conj(np.swapaxes(got, -1, -2)) - np.eye(3)).max() < 1e-13


def test_rk3_is_third_order(oracle):
    """Error at fixed t against a fine-step run: halving eps divides it by 8."""
    n = (4, 4, 4, 4)
    U0 = oracle.gen_expiah(n, 0.3, 11, 0)

    def plaq_at(eps, t=0.16):
        U = U0.copy()
        steps = int(round(t / eps))
        rows = oracle.flow(U, n, eps, steps, steps)  # measured at t = 0 and after the last step
        assert abs(rows[-1, 1] - t) < 1e-9
        return rows[-1, 2]

    fine = plaq_at(0.0025)
    errs = [abs(plaq_at(e) - fine) for e in (0.04, 0.02, 0.01)]
    ratios = [errs[0] / errs[1], errs[1] / errs[2]]
    print("errors", errs, "ratios", ratios)
    assert all(6.0 < r < 10.0 for r in ratios)


def test_flow_raises_the_plaquette(oracle):
    """The Wilson flow is a gradient flow of the action: the plaquette grows."""
    n = (4, 4, 4, 4)
    U = oracle.gen_expiah(n, 0.35, 3, 0)
    rows = oracle.flow(U, n, 0.02, 40, 1)
    assert np.all(np.diff(rows[:, 2]) > 0)


def _cplx(a):
    """(..., 18) doubles, row-major (re, im) -> (..., 3, 3) complex."""
    return (a[..., 0::2] + 1j * a[..., 1::2]).reshape(a.shape[:-1] + (3, 3))


@pytest.mark.parametrize("n", [(4, 4, 4, 4), (3, 4, 5, 6)])
def test_plaquette_field_form_of_the_force(oracle, n):
    """The identity the two-kernel stage computes:
    D_mu(x) = sum_{nu != mu} s_{mu nu} [H_p(x) - U_nu(x-nu)^+ H_p(x-nu) U_nu(x-nu)],
    with H_p = (i/2)[P_p - P_p^+]_TL of the plaquette P_ab(x) = U_a(x) U_b(x+a)
    U_a(x+b)^+ U_b(x)^+ (a < b) and s = +1 for mu < nu, -1 otherwise, against the
    oracle's staple form of the reference's computeDerivative, in FP64."""
    U = _cplx(oracle.gen_expiah(n, 0.4, 3))  # (t, z, y, x, mu, 3, 3)
    axis = {0: 3, 1: 2, 2: 1, 3: 0}  # direction -> array axis (x fastest)

    def up(a, d):  # a(x + d)
        return np.roll(a, -1, axis=axis[d])

    def down(a, d):  # a(x - d)
        return np.roll(a, 1, axis=axis[d])

    dag = lambda m: np.conj(np.swapaxes(m, -1, -2))

    def herm(x):  # (i/2)[X - X^+]_TL
        a = x - dag(x)
        a = a - np.trace(a, axis1=-2, axis2=-1)[..., None, None] / 3 * np.eye(3)
        return 0.5j * a

    planes = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    H = {}
    for a, b in planes:
        ua, ub = U[..., a, :, :], U[..., b, :, :]
        H[a, b] = herm(ua @ up(ub, a) @ dag(up(ua, b)) @ dag(ub))
    for mu in range(4):
        d = 0
        for nu in range(4):
            if nu == mu:
                continue
            h = H[min(mu, nu), max(mu, nu)]
            v = down(U[..., nu, :, :], nu)
            d = d + (1 if mu < nu else -1) * (h - dag(v) @ down(h, nu) @ v)
        want = _cplx(oracle.derivative(oracle_field(U, n), n, mu)).reshape(d.shape)
        assert np.abs(d - want).max() < 1e-13, mu


def oracle_field(Uc, n):
    """(t, z, y, x, mu, 3, 3) complex -> the oracle's (t, z, y, x, mu, 18) doubles."""
    out = np.empty(Uc.shape[:-2] + (18,))
    out[..., 0::2] = Uc.real.reshape(Uc.shape[:-2] + (9,))
    out[..., 1::2] = Uc.imag.reshape(Uc.shape[:-2] + (9,))
    return np.ascontiguousarray(out)
