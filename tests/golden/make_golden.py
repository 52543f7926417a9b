"""Generates tests/golden/element_kat.json.

Known-answer values for the element-level routines, computed by an
independent numpy restatement written directly from the reference sources
(it does not call the oracle or the product):
  * SolveFem::Hex8Isoparametric (SolveFem.cpp:339-408): Ndiff rows as written
    at :390-395, Jacobian, inverse, B (6 x 24) laid out as at :400, D at
    :370-376, ke += W_i W_j W_k B'DB det(J) over the rounded 3-point rule.
  * SolveFem::ComputeVolOfHex (SolveFem.cpp:423-467), 5 tets.
  * PDEFilter::KeHel (PDEFilter.cpp:185-240) for hex8 and tet4/KeHel.cpp.
  * SolveFem::Tet4Isoparametric (tet4/Tet4Isoparametric.cpp).
and the boundary-condition fixture counts of the reference's mesh/ folder
(fixeddofs.txt, loaddof_1.txt, load_1.txt), read when the reference tree is
present.

    python tests/golden/make_golden.py [reference_root]
"""
import json
import os
import shutil
import sys

import numpy as np

G = [-0.775, 0.0, 0.775]
W = [0.556, 0.889, 0.556]


def D_matrix(nu):
    lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = 1.0 / (2.0 * (1.0 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[0, 0] = D[1, 1] = D[2, 2] = lam + 2 * mu
    D[3, 3] = D[4, 4] = D[5, 5] = mu
    return D


def ndiff_hex(xi, eta, zeta):
    # rows exactly as written in SolveFem.cpp (diagonal numbering)
    r0 = [-0.125 * (zeta - 1) * (eta - 1), 0.125 * (zeta - 1) * (eta - 1), 0.125 * (zeta - 1) * (eta + 1),
          -0.125 * (zeta - 1) * (eta + 1), 0.125 * (zeta + 1) * (eta - 1), -0.125 * (zeta + 1) * (eta - 1),
          -0.125 * (zeta + 1) * (eta + 1), 0.125 * (zeta + 1) * (eta + 1)]
    r1 = [-0.125 * (zeta - 1) * (xi - 1), 0.125 * (zeta - 1) * (xi + 1), 0.125 * (zeta - 1) * (xi - 1),
          -0.125 * (zeta - 1) * (xi + 1), 0.125 * (zeta + 1) * (xi - 1), -0.125 * (zeta + 1) * (xi + 1),
          -0.125 * (zeta + 1) * (xi - 1), 0.125 * (zeta + 1) * (xi + 1)]
    r2 = [-0.125 * (xi - 1) * (eta - 1), 0.125 * (xi + 1) * (eta - 1), 0.125 * (xi - 1) * (eta + 1),
          -0.125 * (xi + 1) * (eta + 1), 0.125 * (xi - 1) * (eta - 1), -0.125 * (xi + 1) * (eta - 1),
          -0.125 * (xi - 1) * (eta + 1), 0.125 * (xi + 1) * (eta + 1)]
    return np.array([r0, r1, r2])


def B_matrix(dN):
    n = dN.shape[1]
    z = np.zeros(n)
    return np.array([np.concatenate([dN[0], z, z]), np.concatenate([z, dN[1], z]), np.concatenate([z, z, dN[2]]),
                     np.concatenate([dN[1], dN[0], z]), np.concatenate([z, dN[2], dN[1]]),
                     np.concatenate([dN[2], z, dN[0]])])


def hex8_ke(co, nu=0.3):
    D = D_matrix(nu)
    ke = np.zeros((24, 24))
    for i in range(3):
        for j in range(3):
            for k in range(3):
                Nd = ndiff_hex(G[i], G[j], G[k])
                J = Nd @ co
                dN = np.linalg.inv(J) @ Nd
                B = B_matrix(dN)
                ke += W[i] * W[j] * W[k] * B.T @ D @ B * np.linalg.det(J)
    return ke


def hex8_vol(co):
    def tet(a, b, c, d):
        return 1.0 / 6.0 * np.dot(co[a] - co[b], np.cross(co[a] - co[c], co[a] - co[d]))
    p1 = tet(5, 0, 1, 3)
    p2 = tet(6, 0, 3, 2)
    p3 = 1.0 / 6.0 * np.dot(co[0] - co[5], np.cross(co[0] - co[4], co[0] - co[6]))
    p4 = 1.0 / 6.0 * np.dot(co[3] - co[5], np.cross(co[3] - co[6], co[3] - co[7]))
    p5 = 1.0 / 6.0 * np.dot(co[5] - co[0], np.cross(co[5] - co[3], co[5] - co[6]))
    return abs(p1) + abs(p2) + abs(p3) + abs(p4) + abs(p5)


def hex8_kehel(co, rmin):
    r = 1 / (2 * np.sqrt(3)) * rmin
    Kd = np.eye(3) * r * r
    KE = np.zeros((8, 8))
    T = np.zeros(8)
    for i in range(3):
        for j in range(3):
            for k in range(3):
                s, t, v = G[i], G[j], G[k]
                N = np.array([(1 - s) * (1 - t) * (1 - v), (1 + s) * (1 - t) * (1 - v), (1 - s) * (1 + t) * (1 - v),
                              (1 + s) * (1 + t) * (1 - v), (1 - s) * (1 - t) * (1 + v), (1 + s) * (1 - t) * (1 + v),
                              (1 - s) * (1 + t) * (1 + v), (1 + s) * (1 + t) * (1 + v)]) * 0.125
                dN = np.array([
                    [-(1 - t) * (1 - v), (1 - t) * (1 - v), -(1 + t) * (1 - v), (1 + t) * (1 - v),
                     -(1 - t) * (1 + v), (1 - t) * (1 + v), -(1 + t) * (1 + v), (1 + t) * (1 + v)],
                    [-(1 - s) * (1 - v), -(1 + s) * (1 - v), (1 - s) * (1 - v), (1 + s) * (1 - v),
                     -(1 - s) * (1 + v), -(1 + s) * (1 + v), (1 - s) * (1 + v), (1 + s) * (1 + v)],
                    [-(1 - s) * (1 - t), -(1 + s) * (1 - t), -(1 - s) * (1 + t), -(1 + s) * (1 + t),
                     (1 - s) * (1 - t), (1 + s) * (1 - t), (1 - s) * (1 + t), (1 + s) * (1 + t)]]) * 0.125
                J = dN @ co
                Dn = np.linalg.inv(J) @ dN
                w = W[i] * W[j] * W[k]
                KE += w * (Dn.T @ Kd @ Dn + np.outer(N, N)) * np.linalg.det(J)
                T += w * N * np.linalg.det(J)
    return KE, T


def tet4_ke(co, nu=0.3):
    Nd = np.array([[-1.0, 1, 0, 0], [-1.0, 0, 1, 0], [-1.0, 0, 0, 1]])
    J = Nd @ co
    detJ = np.sqrt(np.linalg.det(Nd @ co @ co.T @ Nd.T))
    dN = np.linalg.inv(J) @ Nd
    B = B_matrix(dN)
    return 1.0 / 6.0 * B.T @ D_matrix(nu) @ B * detJ


def tet4_kehel(co, rmin):
    r = 1 / (2 * np.sqrt(3)) * rmin
    Kd = np.eye(3) * r * r
    a = (5.0 + 3.0 * np.sqrt(5.0)) / 20.0
    b = (5.0 - np.sqrt(5.0)) / 20.0
    Gp = [[a, b, b], [b, a, b], [b, b, a], [b, b, b]]
    dN = np.array([[-1.0, 1, 0, 0], [-1.0, 0, 1, 0], [-1.0, 0, 0, 1]])
    J = dN @ co
    Dn = np.linalg.inv(J) @ dN
    KE = np.zeros((4, 4))
    T = np.zeros(4)
    for s, t, v in Gp:
        N = np.array([1 - s - t - v, s, t, v])
        KE += 1.0 / 24.0 * (Dn.T @ Kd @ Dn + np.outer(N, N)) * np.linalg.det(J)
        T += 1.0 / 24.0 * N * np.linalg.det(J)
    return KE, T


def cases():
    unit = np.array([[(l & 1), (l >> 1) & 1, (l >> 2) & 1] for l in range(8)], float)
    rng = np.random.default_rng(7)
    jit = unit * np.array([1.3, 0.8, 1.1]) + rng.uniform(-0.1, 0.1, (8, 3))
    tunit = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    tjit = tunit + rng.uniform(-0.15, 0.15, (4, 3))
    return {"hex_unit": unit, "hex_jitter": jit, "tet_unit": tunit, "tet_jitter": tjit}


def main():
    """usage: make_golden.py REFERENCE_ROOT (or TOPO_REFERENCE_ROOT in the environment): the checkout of the
    reference whose mesh/ boundary-condition files are copied into tests/golden/reference_mesh/"""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TOPO_REFERENCE_ROOT")
    if not ref:
        sys.exit("usage: make_golden.py REFERENCE_ROOT (or set TOPO_REFERENCE_ROOT)")
    out = {"nu": 0.3, "rmin": 1.5, "cases": {}}
    for name, co in cases().items():
        rec = {"coords": co.tolist()}
        if name.startswith("hex"):
            ke = hex8_ke(co)
            kh, T = hex8_kehel(co, 1.5)
            rec.update(ke=ke.tolist(), kehel=kh.tolist(), T=T.tolist(), vol=hex8_vol(co))
        else:
            ke = tet4_ke(co)
            kh, T = tet4_kehel(co, 1.5)
            rec.update(ke=ke.tolist(), kehel=kh.tolist(), T=T.tolist(),
                       vol=abs(np.linalg.det(np.array([co[1] - co[0], co[2] - co[0], co[3] - co[0]]))) / 6.0)
        out["cases"][name] = rec
    mesh = os.path.join(ref, "mesh")
    if os.path.isdir(mesh):
        fixed = np.loadtxt(os.path.join(mesh, "fixeddofs.txt"), dtype=np.int64).ravel()
        ld = np.loadtxt(os.path.join(mesh, "loaddof_1.txt"), dtype=np.int64).ravel()
        lv = np.loadtxt(os.path.join(mesh, "load_1.txt")).ravel()
        trip = fixed.reshape(-1, 3)
        out["reference_fixtures"] = {
            "n_fixed": int(fixed.size),
            "fixed_triples": bool(np.all(trip == trip[:, :1] + np.arange(3)) and np.all(trip[:, 0] % 3 == 0)),
            "n_fixed_nodes": int(fixed.size // 3), "n_load": int(ld.size),
            "load_dofs_mod3": sorted(set(int(x) for x in ld % 3)), "load_values": sorted(set(float(x) for x in lv)),
            "lattice": [140, 70, 40]}
        # the reference's own boundary-condition files, byte for byte, so that
        # tests can read them through the library's mesh reader where the
        # reference checkout is absent
        dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_mesh")
        os.makedirs(dst, exist_ok=True)
        for name in ("fixeddofs.txt", "loaddof_1.txt", "load_1.txt"):
            shutil.copyfile(os.path.join(mesh, name), os.path.join(dst, name))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "element_kat.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
