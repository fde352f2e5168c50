"""Gauge covariance of the device path at lattice sizes the oracle does not
reach: under U_mu(x) -> G(x) U_mu(x) G(x+mu)^+ with random G(x) in SU(3),
the observables are unchanged and the flow commutes with the transformation
(the force transforms as G Z G^+, so does e^{iQ})."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def to_c(U):
    a = U.reshape(U.shape[:-1] + (3, 3, 2))
    return a[..., 0] + 1j * a[..., 1]


def to_r(C):
    return np.stack([C.real, C.imag], axis=-1).reshape(C.shape[:-2] + (18,))


def random_su3(shape, rng):
    z = (rng.standard_normal(shape + (3, 3)) + 1j * rng.standard_normal(shape + (3, 3))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r, axis1=-2, axis2=-1)
    q = q * (d / np.abs(d))[..., None, :]
    det = np.linalg.det(q)
    q[..., 0, :] /= det[..., None]  # det 1: one row takes the phase
    return q


def transform(U, G):
    """U shape (t, z, y, x, mu, 18); G shape (t, z, y, x, 3, 3)."""
    C = to_c(U)
    out = np.empty_like(C)
    axis = {0: 3, 1: 2, 2: 1, 3: 0}  # direction -> array axis (x fastest)
    for mu in range(4):
        Gp = np.roll(G, -1, axis=axis[mu])  # G(x + mu)
        out[..., mu, :, :] = G @ C[..., mu, :, :] @ np.conj(np.swapaxes(Gp, -1, -2))
    return to_r(out)


@pytest.mark.parametrize("precision,n", [("fp64", (16, 16, 16, 16)), ("fp64", (12, 8, 10, 14)),
                                         ("fp32_18", (16, 16, 16, 16)), ("fp32_12", (16, 16, 16, 16))])
def test_observables_invariant_and_flow_covariant(precision, n):
    from latticeyangmills_b200 import GluonField

    rng = np.random.default_rng(2024)
    with GluonField(n, "fp64") as f:
        f.init_links("expiah", 0.35, 99)
        U = f.download()
    G = random_su3((n[3], n[2], n[1], n[0]), rng)
    Ug = transform(U, G)
    tol_obs = 1e-12 if precision == "fp64" else 2e-6
    tol_link = 1e-12 if precision == "fp64" else 5e-5
    res = {}
    for name, field in (("plain", U), ("gauged", Ug)):
        with GluonField(n, precision) as f:
            f.upload(field)
            rows = f.flow(0.02, 10, 5, reunit_every=5 if precision != "fp64" else 0)
            res[name] = (rows, f.download())
    (r0, V0), (r1, V1) = res["plain"], res["gauged"]
    # plaquette, topological charge, energy and t^2 E of every measured row
    np.testing.assert_allclose(r1[:, [2, 4, 5]], r0[:, [2, 4, 5]], rtol=tol_obs)
    assert np.abs(r1[:, 3] - r0[:, 3]).max() < tol_obs * max(1.0, np.abs(r0[:, 3]).max()) * 10
    # flow(G U) = G flow(U): compare the transported flowed field
    diff = np.abs(transform(V0, G) - V1).max()
    print(precision, n, "max |G V G+ - V_g|", diff)
    assert diff < tol_link
