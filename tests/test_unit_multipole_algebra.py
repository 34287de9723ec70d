"""The algebra of the P2M factored through unit-density multipoles, on the
host: every column's node weights (the seven kinds of the image plan, the
first four also the free-space passes) are linear in the six density
components of the node's triangle, and the unit columns formed from the 26
node moments (the combinations coded in k_p2m_unit / k_p2m_unit_f) reproduce
sum_nodes F_node . weights_node for random features, nodes, normals, Lame
constants and densities."""
import numpy as np
import pytest


def node_weights(kind, sl, dl, nn, y, lam, mu):
    # the weights of one node (charge, dipole x/y/z, quadrupole xx-zz, yy-zz,
    # 2xy, 2xz, 2yz) per column kind, as img_node_weights / k_p2m_weights
    al = (lam + mu) / (lam + 2 * mu)
    c1, c2, inv2mu = 2 - al, (2 * lam + 3 * mu) / (lam + 2 * mu), 1 / (2 * mu)
    wv = np.zeros(9)
    Q = np.zeros((3, 3))
    dln = dl @ nn
    T = lam * dln * np.eye(3) + mu * (np.outer(dl, nn) + np.outer(nn, dl))
    h = -y[2]
    if kind < 3:
        wv[0] = sl[kind] * inv2mu
        wv[1:4] = 0.5 * (nn * dl[kind] + dl * nn[kind])
    elif kind == 3:
        wv[0] = (sl @ y) * c1 * inv2mu + dln * c2
        wv[1:4] = 0.5 * c1 * (nn * (dl @ y) + dl * (nn @ y))
    elif kind == 4:
        wv[0] = -(2 - al) * sl[2]
        wv[1:4] = -h * al * sl - (2 - 2 * al) * T[2]
        Q = -h * al * T
    elif kind == 5:
        wv[1:4] = -sl
        Q = -T
    else:
        wv[1:4] = [sl[0], sl[1], -sl[2]]
        Q[0, 0], Q[1, 1], Q[2, 2] = T[0, 0], T[1, 1], -T[2, 2]
        Q[0, 1] = Q[1, 0] = T[0, 1]
    wv[4:] = [Q[0, 0] - Q[2, 2], Q[1, 1] - Q[2, 2], 2 * Q[0, 1], 2 * Q[0, 2], 2 * Q[1, 2]]
    return wv


def unit_columns(M0, M1, nn, lam, mu):
    # H[kind][s] from the moments M0[row] = sum w F[row], M1[e][row] = sum w y_e F[row]
    al = (lam + mu) / (lam + 2 * mu)
    c1, c2, inv2mu = 2 - al, (2 * lam + 3 * mu) / (lam + 2 * mu), 1 / (2 * mu)
    H = np.zeros((7, 6), dtype=complex)
    nd = nn @ M0[1:4]
    for p in range(3):
        H[p, p] = inv2mu * M0[0]
        for e in range(3):
            H[p, 3 + e] = 0.5 * ((nd if e == p else 0) + nn[p] * M0[1 + e])
    for e in range(3):
        H[3, e] = c1 * inv2mu * M1[e][0]
        H[3, 3 + e] = c2 * nn[e] * M0[0] + 0.5 * c1 * (sum(nn[d] * M1[e][1 + d] for d in range(3))
                                                      + sum(nn[d] * M1[d][1 + e] for d in range(3)))
    for e in range(3):
        E = np.zeros(3)
        E[e] = 1
        Te = lam * nn[e] * np.eye(3) + mu * (np.outer(E, nn) + np.outer(nn, E))
        qv = np.array([Te[0, 0] - Te[2, 2], Te[1, 1] - Te[2, 2], 2 * Te[0, 1], 2 * Te[0, 2], 2 * Te[1, 2]])
        qu = np.array([Te[0, 0] + Te[2, 2], Te[1, 1] + Te[2, 2], 2 * Te[0, 1], 0, 0])
        H[4, e] = al * M1[2][1 + e] - ((2 - al) * M0[0] if e == 2 else 0)
        H[4, 3 + e] = -(2 - 2 * al) * (Te[2] @ M0[1:4]) + al * (qv @ M1[2][4:9])
        H[5, e] = -M0[1 + e]
        H[5, 3 + e] = -(qv @ M0[4:9])
        H[6, 3 + e] = qu @ M0[4:9]
    H[6, 0:3] = [M0[1], M0[2], -M0[3]]
    return H


@pytest.mark.parametrize("seed", range(5))
def test_unit_columns_reproduce_node_sums(seed):
    rng = np.random.default_rng(seed)
    lam, mu = rng.uniform(0.5, 2.0), rng.uniform(0.3, 1.5)
    nn = rng.normal(size=3)
    nn /= np.linalg.norm(nn)
    nodes = 12
    F = rng.normal(size=(nodes, 9)) + 1j * rng.normal(size=(nodes, 9))
    w = rng.uniform(0.01, 1.0, nodes)
    Y = rng.normal(size=(nodes, 3)) * 5.0 - np.array([0, 0, 10.0])
    M0 = (w[:, None] * F).sum(0)
    M1 = np.array([(w[:, None] * Y[:, e:e + 1] * F).sum(0) for e in range(3)])
    H = unit_columns(M0, M1, nn, lam, mu)
    for _ in range(4):
        sig = rng.normal(size=6)
        for kind in range(7):
            ref = sum(F[i] @ (w[i] * node_weights(kind, sig[:3], sig[3:], nn, Y[i], lam, mu)) for i in range(nodes))
            got = H[kind] @ sig
            assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref))
