"""The oracle (CPU restatement) pinned against the golden known-answer values
and an independent scipy restatement.  CPU only."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from conftest import rel

HEX_CASES = ["hex_unit", "hex_jitter"]
TET_CASES = ["tet_unit", "tet_jitter"]


@pytest.mark.parametrize("case", HEX_CASES)
def test_hex8_element_kat(O, golden, case):
    g = golden["cases"][case]
    co = np.array(g["coords"])
    ke = O.hex8_ke(co, golden["nu"])
    assert rel(ke, g["ke"]) < 1e-14
    kh, T = O.hex8_kehel(co, golden["rmin"])
    assert rel(kh, g["kehel"]) < 1e-14
    assert rel(T, g["T"]) < 1e-14
    assert abs(O.hex8_volume(co) - g["vol"]) < 1e-14


def test_hex8_known_values(O):
    """Derived values of SolveFem.cpp:339-408 on the unit cube."""
    co = np.array([[(l & 1), (l >> 1) & 1, (l >> 2) & 1] for l in range(8)], float)
    ke = O.hex8_ke(co)
    assert abs(ke[0, 0] - 0.23555343219393224) < 1e-15
    assert abs(ke[0, 1] - (-0.10711282824086732)) < 1e-15
    assert abs(ke[0, 8] - 0.08027537747066561) < 1e-15
    assert np.abs(ke - ke.T).max() < 1e-16
    w = np.sort(np.abs(np.linalg.eigvalsh(ke)))
    assert np.all(w[:6] < 1e-15) and w[6] > 0.06  # 6 rigid-body modes
    _, T = O.hex8_kehel(co, 1.5)
    assert abs(T.sum() - 2.001 ** 3 / 8) < 1e-14  # rounded weights sum to 2.001
    assert abs(O.hex8_volume(co) - 1.0) < 1e-15


@pytest.mark.parametrize("case", TET_CASES)
def test_tet4_element_kat(O, golden, case):
    g = golden["cases"][case]
    co = np.array(g["coords"])
    assert rel(O.tet4_ke(co, golden["nu"]), g["ke"]) < 1e-14
    kh, T = O.tet4_kehel(co, golden["rmin"])
    assert rel(kh, g["kehel"]) < 1e-14
    assert rel(T, g["T"]) < 1e-14
    assert abs(O.tet4_volume(co) - g["vol"]) < 1e-14


def test_reference_bc_fixture_counts(O, golden):
    """The generator's lattice-index BCs reproduce the counts of the reference
    fixtures mesh/fixeddofs.txt (8733 = 3 x 71 x 41) and mesh/loaddof_1.txt
    (41 DOFs, all 3n+1, value 1) on the 140 x 70 x 40 lattice."""
    fx = golden.get("reference_fixtures")
    if fx is None:
        pytest.skip("reference fixture summary not recorded")
    nx, ny, nz = fx["lattice"]
    f, ld, lv = O.cantilever_bcs(nx, ny, nz, load_mode=1)
    assert f.size == fx["n_fixed"] and fx["fixed_triples"]
    assert np.all(f.reshape(-1, 3) == f.reshape(-1, 3)[:, :1] + np.arange(3))
    assert ld.size == fx["n_load"]
    assert sorted(set((ld % 3).tolist())) == fx["load_dofs_mod3"]
    assert sorted(set(lv.tolist())) == fx["load_values"]


def test_tet_split_positive():
    import oracle.oracle as O
    v = O.lattice_nodes(6, 4, 3, 1.0, 0.2, True, 2024)
    e, bad = O.tet4_elements(6, 4, 3, v)
    assert bad == 0 and e.shape == (6 * 4 * 3 * 6, 4)
    vol = [O.tet4_volume(v[t]) for t in e]
    assert abs(sum(vol) - 6 * 4 * 3) < 1e-9  # tets tile the box (interior jitter only)


@pytest.fixture(scope="module")
def small(O):
    v, e, f, ld, lv = O.cantilever(12, 6, 4)
    return v, e, f, ld, lv


def test_assembly_matches_scipy(O, small):
    """Assembled K (MatZeroRowsColumns identity) equals an independent scipy
    assembly from the element matrices."""
    v, e, f, ld, lv = small
    orc = O.Oracle(v, e, f, ld, lv, Emax=1.0, rmin=1.5)
    rng = np.random.default_rng(1)
    x = rng.uniform(0.01, 1, e.shape[0])
    orc.assemble(x)
    K = orc.csr()
    rows, cols, vals = [], [], []
    for el in range(e.shape[0]):
        ke = orc.element_ke(el)
        dofs = np.concatenate([3 * e[el], 3 * e[el] + 1, 3 * e[el] + 2])
        E = 1e-9 + x[el] ** 3 * (1 - 1e-9)
        rows.append(np.repeat(dofs, 24)); cols.append(np.tile(dofs, 24)); vals.append((E * ke).ravel())
    n = 3 * v.shape[0]
    Kr = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n)).tolil()
    for d in f:
        Kr[d, :] = 0
        Kr[:, d] = 0
        Kr[d, d] = 1
    Kr = Kr.tocsr()
    assert abs(K - Kr).max() < 1e-13
    u = rng.standard_normal(n)
    assert rel(orc.kmatvec(u), Kr @ u) < 1e-14


def test_solve_matches_direct(O, small):
    v, e, f, ld, lv = small
    orc = O.Oracle(v, e, f, ld, lv, Emax=1.0, rmin=1.5, fem_rtol=1e-12)
    x = np.full(e.shape[0], 0.3)
    fx, gx, df, dg, U = orc.fem_obj_sens(x, return_u=True)
    K = orc.csr()
    Ud = spl.spsolve(K.tocsc(), orc.rhs())
    assert rel(U, Ud) < 1e-10
    assert abs(fx - orc.rhs() @ Ud) / abs(fx) < 1e-10  # compliance = F.U
    # dg = vol / TV, gx = sum x vol / TV - volfrac
    tv, vol = orc.total_volume()
    assert rel(dg[0], vol / tv) < 1e-15
    assert abs(gx[0] - (0.3 - 0.12)) < 1e-14


def test_filter_matches_direct(O, small):
    """Filter = clamp(TFX' KF^-1 TF x) against a scipy direct solve."""
    v, e, f, ld, lv = small
    orc = O.Oracle(v, e, f, ld, lv, Emax=1.0, rmin=1.5, filter_rtol=1e-13)
    nn, ne = v.shape[0], e.shape[0]
    rows, cols, vals, trow, tcol, tval = [], [], [], [], [], []
    for el in range(ne):
        kh, T = O.hex8_kehel(v[e[el]], 1.5)
        rows.append(np.repeat(e[el], 8)); cols.append(np.tile(e[el], 8)); vals.append(kh.ravel())
        trow.append(e[el]); tcol.append(np.full(8, el)); tval.append(T)
    KF = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(nn, nn))
    TF = sp.csr_matrix((np.concatenate(tval), (np.concatenate(trow), np.concatenate(tcol))), shape=(nn, ne))
    TFX = sp.csr_matrix((np.full(8 * ne, 1 / 8), (np.concatenate(trow), np.concatenate(tcol))), shape=(nn, ne))
    x = np.random.default_rng(2).uniform(0, 1, ne)
    ref = np.clip(TFX.T @ spl.spsolve(KF.tocsc(), TF @ x), 0.01, 1.0)
    assert rel(orc.filter(x, 0.01), ref) < 1e-10


def _mma_py(x, dfdx, gx, dgdx, xmin, xmax, state):
    """Plain-Python restatement of MMA::Update for m = 1 (MMA.cpp:483-969),
    for small n only."""
    import math
    n = len(x)
    state["k"] += 1
    k = state["k"]
    L, U, xo1, xo2 = state["L"], state["U"], state["xo1"], state["xo2"]
    for i in range(n):
        if k < 3:
            L[i] = x[i] - 0.5 * xmax[i] + 0.5 * xmin[i]
            U[i] = x[i] + 0.5 * xmax[i] - 0.5 * xmin[i]
        else:
            h = (x[i] - xo1[i]) * (xo1[i] - xo2[i])
            gam = 0.7 if h < 0 else (1.2 if h > 0 else 1.0)
            L[i] = x[i] - gam * (xo1[i] - L[i])
            U[i] = x[i] + gam * (U[i] - xo1[i])
            xmi = max(1e-5, xmax[i] - xmin[i])
            L[i] = min(max(L[i], x[i] - 10 * xmi), x[i] - 0.01 * xmi)
            U[i] = min(max(U[i], x[i] + 0.01 * xmi), x[i] + 10 * xmi)
    alf = [max(xmin[i], 0.9 * L[i] + 0.1 * x[i]) for i in range(n)]
    bet = [min(xmax[i], 0.9 * U[i] + 0.1 * x[i]) for i in range(n)]
    p0, q0, p1, q1 = [], [], [], []
    for i in range(n):
        d = dfdx[i]
        p0.append((U[i] - x[i]) ** 2 * (max(0, d) + 0.001 * abs(d) + 0.5e-6 / (U[i] - L[i])))
        q0.append((x[i] - L[i]) ** 2 * (max(0, -d) + 0.001 * abs(d) + 0.5e-6 / (U[i] - L[i])))
        g = dgdx[i]
        p1.append((U[i] - x[i]) ** 2 * max(0, g))
        q1.append((x[i] - L[i]) ** 2 * max(0, -g))
    b = sum(p1[i] / (U[i] - x[i]) + q1[i] / (x[i] - L[i]) for i in range(n)) - gx
    state["xo2"], state["xo1"] = list(xo1), list(x)
    lam, mu = 500.0, 1.0
    xv = list(x)

    def xyz(lam):
        lam = max(lam, 0.0)
        y = max(0.0, lam - 1000.0)
        z = 0.0
        for i in range(n):
            pj, qj = p0[i] + p1[i] * lam, q0[i] + q1[i] * lam
            v = (math.sqrt(pj) * L[i] + math.sqrt(qj) * U[i]) / (math.sqrt(pj) + math.sqrt(qj))
            xv[i] = min(max(v, alf[i]), bet[i])
        return lam, y, z

    tol, epsi, err = 1e-9 * math.sqrt(1 + n), 1.0, 1.0
    while epsi > tol:
        loop = 0
        while err > 0.9 * epsi and loop < 100:
            loop += 1
            lam, y, z = xyz(lam)
            grad = sum(p1[i] / (U[i] - xv[i]) + q1[i] / (xv[i] - L[i]) for i in range(n)) - b - y
            grad = -grad - epsi / lam
            H = 0.0
            for i in range(n):
                pj, qj = p0[i] + p1[i] * lam, q0[i] + q1[i] * lam
                PQ = p1[i] / (U[i] - xv[i]) ** 2 - q1[i] / (xv[i] - L[i]) ** 2
                df2 = -1.0 / (2 * pj / (U[i] - xv[i]) ** 3 + 2 * qj / (xv[i] - L[i]) ** 3)
                xp = (math.sqrt(pj) * L[i] + math.sqrt(qj) * U[i]) / (math.sqrt(pj) + math.sqrt(qj))
                if xp < alf[i] or xp > bet[i]:
                    df2 = 0.0
                H += PQ * df2 * PQ
            if lam > 1000.0:
                H -= 1.0
            H -= mu / lam
            corr = 1e-4 * H
            if -corr < 1e-7:
                corr = -1e-7
            H += corr
            s0 = grad / H
            s1 = -mu + epsi / lam - s0 * mu / lam
            theta = 1.005
            theta = max(theta, -1.01 * s0 / lam)
            theta = max(theta, -1.01 * s1 / mu)
            theta = 1.0 / theta
            lam, mu = lam + theta * s0, mu + theta * s1
            lam, y, z = xyz(lam)
            r1 = sum(p1[i] / (U[i] - xv[i]) + q1[i] / (xv[i] - L[i]) for i in range(n)) - b - y + mu
            r2 = mu * lam - epsi
            err = max(abs(r1), abs(r2))
        epsi *= 0.1
    return xv


def test_mma_matches_python_restatement(O):
    """Three successive MMA updates (k < 3 and k > 2 asymptote branches) of the
    C oracle against a plain-Python restatement on a small problem."""
    v, e, f, ld, lv = O.cantilever(4, 2, 2)
    orc = O.Oracle(v, e, f, ld, lv, Emax=1.0, rmin=1.5)
    n = e.shape[0]
    rng = np.random.default_rng(3)
    x = rng.uniform(0.1, 0.9, n)
    state = {"k": 0, "L": [0.0] * n, "U": [0.0] * n, "xo1": [0.0] * n, "xo2": [0.0] * n}
    xp = list(x)
    for it in range(3):
        df = -rng.uniform(0.5, 2.0, n)
        dg = np.full(n, 1.0 / n)
        gx = np.array([float(np.mean(x)) - 0.3])
        xmn, xmx = orc.mma_movelimit(x)
        xn = orc.mma_update(x, df, gx, dg, xmn, xmx)
        xpn = _mma_py(list(xp), list(df), gx[0], list(dg), list(xmn), list(xmx), state)
        assert rel(xn, xpn) < 1e-10, it
        x, xp = xn, xpn


def test_design_change_and_movelimit(O):
    v, e, f, ld, lv = O.cantilever(4, 2, 2)
    orc = O.Oracle(v, e, f, ld, lv)
    x = np.linspace(0.0, 1.0, e.shape[0])
    xmn, xmx = orc.mma_movelimit(x, 0.01, 1.0, 0.2)
    assert np.allclose(xmx, np.minimum(1.0, x + 0.2)) and np.allclose(xmn, np.maximum(0.01, x - 0.2))
    xo = x[::-1].copy()
    ch, xo2 = orc.mma_design_change(x, xo)
    assert ch == np.abs(x - x[::-1]).max() and np.array_equal(xo2, x)


def test_heaviside_continuation_and_projected_sens(O, small):
    """Heaviside projection with the reference's beta continuation
    (PDEFilter.cpp:242-290: beta0 while itr < 30, then on every tenth
    iteration beta = min(betamax, previous beta + 1), clamp at Xmin) and the
    chain rule of ComputeProjectedSens (PDEFilter.cpp:292-341), restated in
    numpy, against the oracle over a 0..75 iteration sequence; the projected
    sensitivity is also checked against a central difference of the
    projection."""
    v, e, f, ld, lv = small
    orc = O.Oracle(v, e, f, ld, lv, Emax=1.0, rmin=1.5)
    rng = np.random.default_rng(5)
    x0, beta0, betamax, Xmin = 0.5, 1.0, 8.0, 0.01
    beta, prev = beta0, beta0
    ne = e.shape[0]
    for itr in range(76):
        xf = rng.uniform(0.0, 1.0, ne)
        if itr < 30:
            beta = beta0
        elif itr % 10 == 0:
            beta = min(betamax, prev + 1.0)
        den = np.tanh(beta * x0) + np.tanh(beta * (1.0 - x0))
        ref = np.maximum((np.tanh(beta * x0) + np.tanh(beta * (xf - x0))) / den, Xmin)
        prev = beta
        xp = orc.heaviside(xf, itr, x0, beta0, betamax, Xmin, proj=1)
        assert rel(xp, ref) < 1e-14, itr
        df, dg = rng.standard_normal(ne), rng.standard_normal((1, ne))
        pdf, pdg = orc.projected_sens(xf, df, dg, x0)
        dx = beta * (1.0 - np.tanh(beta * (xf - x0)) ** 2) / den
        assert rel(pdf, df * dx) < 1e-14 and rel(pdg, dg * dx) < 1e-14, itr
    # beta reached betamax: 30 -> 2, 40 -> 3, ..., 70 -> 6
    assert beta == 6.0
    h = 1e-6
    xf = rng.uniform(0.3, 0.7, ne)  # away from the Xmin clamp
    up = (np.tanh(beta * x0) + np.tanh(beta * (xf + h - x0))) / den
    dn = (np.tanh(beta * x0) + np.tanh(beta * (xf - h - x0))) / den
    pdf, _ = orc.projected_sens(xf, np.ones(ne), np.ones((1, ne)), x0)
    assert rel(pdf, (up - dn) / (2 * h)) < 1e-7
    # proj = 0 copies the filtered field
    xf = rng.uniform(0.0, 1.0, ne)
    assert np.array_equal(orc.heaviside(xf, 80, x0, beta0, betamax, Xmin, proj=0), xf)
    orc.close()


def test_von_mises_matches_restatement(O):
    """The oracle's element von Mises stress against a numpy restatement of
    stress/ComputeStress.cpp:53-104: strains at the element centre from the
    inverse Jacobian, E = Emax isotropic stress scaled by sqrt(x), and the
    von Mises norm, on jittered elements with random displacements."""
    rng = np.random.default_rng(9)
    nu, Emax = 0.3, 2.5
    lam = nu / ((1 + nu) * (1 - 2 * nu))
    mu = 1 / (2 * (1 + nu))
    D = np.array([[lam + 2 * mu, lam, lam, 0, 0, 0], [lam, lam + 2 * mu, lam, 0, 0, 0],
                  [lam, lam, lam + 2 * mu, 0, 0, 0], [0, 0, 0, mu, 0, 0], [0, 0, 0, 0, mu, 0],
                  [0, 0, 0, 0, 0, mu]])
    # diagonal local numbering: node l at (xi, eta, zeta) = signs of bits 0, 1, 2
    sg = np.array([[1 if l & 1 else -1, 1 if l & 2 else -1, 1 if l & 4 else -1] for l in range(8)], dtype=float)
    Nd = 0.125 * sg.T  # dN/d(xi, eta, zeta) at the centre, 3 x 8
    for _ in range(20):
        co = (sg + 1) / 2 * rng.uniform(0.5, 2.0, 3) + rng.uniform(-0.1, 0.1, (8, 3))
        ue = rng.standard_normal(24)  # [x0..x7, y0..y7, z0..z7]
        x = rng.uniform(0.01, 1.0)
        dN = np.linalg.solve(Nd @ co, Nd)
        z = np.zeros(8)
        B = np.array([np.r_[dN[0], z, z], np.r_[z, dN[1], z], np.r_[z, z, dN[2]],
                      np.r_[dN[1], dN[0], z], np.r_[z, dN[2], dN[1]], np.r_[dN[2], z, dN[0]]])
        s = np.sqrt(x) * Emax * D @ B @ ue
        ref = np.sqrt(0.5 * ((s[0] - s[1]) ** 2 + (s[0] - s[2]) ** 2 + (s[1] - s[2]) ** 2
                             + 6 * (s[3] ** 2 + s[4] ** 2 + s[5] ** 2)))
        assert abs(O.von_mises_hex8(co, nu, Emax, x, ue) - ref) <= 1e-12 * ref
