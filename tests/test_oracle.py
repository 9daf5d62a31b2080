"""CPU oracle pinned by analytic known-answer tests.

The reference ships no CPU dslash and no golden vectors for the hop or the solver
(its only dslash test, tests/test_dslash/test_wilson_dslash.cu:47-101, compares
nothing), so the oracle's conventions are pinned here from the operator definition:
free-field plane waves, gauge covariance, gamma5-hermiticity / adjointness of the
dagger flag, antiperiodic-link equivalence, the reference's projector tables
(include/kernel/complex_matmul.cuh) and M x = b.
"""
import numpy as np
import pytest

from qcu_mrhs_b200 import fields as F

# DeGrand-Rossi gamma matrices (reference include/kernel/qcu_gamma.cuh:10-191 list 1 + gamma_mu)
G = np.zeros((4, 4, 4), dtype=complex)
G[0][0, 3] = 1j; G[0][1, 2] = 1j; G[0][2, 1] = -1j; G[0][3, 0] = -1j
G[1][0, 3] = -1; G[1][1, 2] = 1; G[1][2, 1] = 1; G[1][3, 0] = -1
G[2][0, 2] = 1j; G[2][1, 3] = -1j; G[2][2, 0] = -1j; G[2][3, 1] = 1j
G[3][0, 2] = 1; G[3][1, 3] = 1; G[3][2, 0] = 1; G[3][3, 1] = 1


def test_gamma_basis_is_a_clifford_algebra():
    for a in range(4):
        for b in range(4):
            anti = G[a] @ G[b] + G[b] @ G[a]
            assert np.allclose(anti, 2 * np.eye(4) * (a == b))
        assert np.allclose(G[a], G[a].conj().T)


@pytest.mark.parametrize("L", [(4, 4, 4, 8), (6, 2, 4, 4)])
def test_free_field_plane_wave(oracle_lib, L):
    O = oracle_lib
    nc = 3
    Lx, Ly, Lz, Lt = L
    V = Lx * Ly * Lz * Lt
    vh = V // 2
    n = (1, 1, 3, 2)
    p = [2 * np.pi * n[i] / L[i] for i in range(4)]
    rng = np.random.default_rng(0)
    chi = rng.standard_normal((4, nc)) + 1j * rng.standard_normal((4, nc))
    t, z, y, x = np.meshgrid(np.arange(Lt), np.arange(Lz), np.arange(Ly), np.arange(Lx), indexing="ij")
    phase = np.exp(1j * (p[0] * x + p[1] * y + p[2] * z + p[3] * t))
    lex = (phase[..., None, None] * chi).reshape(V, 4, nc)
    eo = O.fermion_to_eo(lex, L).reshape(2, vh, 4, nc)
    gauge = F.gauge_field(L, nc, 1, kind="unit")
    K = sum(2 * np.cos(p[mu]) * np.eye(4) - 2j * np.sin(p[mu]) * G[mu] for mu in range(4))
    expect = O.fermion_to_eo(np.einsum("ab,vbc->vac", K, lex), L).reshape(2, vh, 4, nc)
    for par in range(2):
        out = O.hop(eo[1 - par][..., None], gauge, L, par)
        assert np.abs(out[..., 0] - expect[par]).max() < 1e-12


def _random_problem(L, nc, m, seed):
    gauge = F.gauge_field(L, nc, seed, kind="haar")
    psi = F.gaussian_fermions(L, nc, m, seed + 100)
    return gauge, psi


def test_gauge_covariance(oracle_lib):
    O = oracle_lib
    L = (4, 4, 2, 6)
    nc, m = 3, 2
    Lx, Ly, Lz, Lt = L
    vh = F.half_volume(L)
    gauge, psi = _random_problem(L, nc, m, 2)
    om = F.haar_sun(np.random.default_rng(3), 2 * vh, nc).reshape(2, vh, nc, nc)

    def fwd(par, idx, mu):
        xh = idx % (Lx // 2); q = idx // (Lx // 2)
        yy = q % Ly; q //= Ly
        zz = q % Lz; tt = q // Lz
        xx = 2 * xh + ((par + yy + zz + tt) & 1)
        c = [xx, yy, zz, tt]
        c[mu] = (c[mu] + 1) % L[mu]
        return ((c[3] * Lz + c[2]) * Ly + c[1]) * (Lx // 2) + c[0] // 2

    g2 = np.empty_like(gauge)
    idx = np.arange(vh)
    for mu in range(4):
        for par in range(2):
            nb = fwd(par, idx, mu)
            g2[mu, par] = om[par] @ gauge[mu, par] @ np.conj(np.swapaxes(om[1 - par][nb], -1, -2))
    for par in range(2):
        inp = F.to_mrhs(psi[:, 1 - par])
        out = O.hop(inp, gauge, L, par)
        out2 = O.hop(np.einsum("vab,vsbm->vsam", om[1 - par], inp), g2, L, par)
        assert np.abs(out2 - np.einsum("vab,vsbm->vsam", om[par], out)).max() < 1e-12


def test_dagger_is_adjoint_and_gamma5_hermitian(oracle_lib):
    O = oracle_lib
    L = (4, 4, 4, 4)
    gauge, psi = _random_problem(L, 3, 2, 4)
    g5 = G[0] @ G[1] @ G[2] @ G[3]
    for par in range(2):
        a = F.to_mrhs(psi[:, 1 - par])
        b = F.to_mrhs(psi[:, par])
        lhs = np.vdot(b, O.hop(a, gauge, L, par))
        rhs = np.vdot(O.hop(b, gauge, L, 1 - par, dagger=True), a)
        assert abs(lhs - rhs) / abs(lhs) < 1e-13
        g5a = np.einsum("ab,vbcm->vacm", g5, a)
        got = np.einsum("ab,vbcm->vacm", g5, O.hop(g5a, gauge, L, par))
        assert np.abs(got - O.hop(a, gauge, L, par, dagger=True)).max() < 1e-13


def test_antiperiodic_boundary_equals_folded_links(oracle_lib):
    O = oracle_lib
    L = (4, 2, 2, 6)
    gauge, psi = _random_problem(L, 3, 3, 5)
    folded = F.fold_t_boundary(gauge, L, -1.0)
    for par in range(2):
        a = F.to_mrhs(psi[:, 1 - par])
        assert np.array_equal(O.hop(a, folded, L, par), O.hop(a, gauge, L, par, t_sign=-1.0))
        assert not np.allclose(O.hop(a, gauge, L, par), O.hop(a, gauge, L, par, t_sign=-1.0))


def _reference_projector_hop(inp, gauge, L, parity, dagger):
    """Hop from the reference's T1/T2 projection and L-reconstruction tables
    (include/kernel/complex_matmul.cuh:16-227 loaders, :503-600 calc_L_from_R;
    forward hop local_dagger = dagger, backward hop local_dagger = !dagger and U^dag,
    include/kernel/su_n_m_rhs_matmul.cuh:312-323)."""
    Lx, Ly, Lz, Lt = L
    vh = F.half_volume(L)
    out = np.zeros_like(inp)
    lxh = Lx // 2
    for idx in range(vh):
        xh = idx % lxh; q = idx // lxh
        y = q % Ly; q //= Ly
        z = q % Lz; t = q // Lz
        eo = (y + z + t) & 1
        for dim in range(4):
            for d in ("fwd", "bwd"):
                c = [xh, y, z, t]
                if dim == 0:
                    if d == "bwd":
                        c[0] = xh + (eo == parity) * (-1 + (xh == 0) * lxh)
                    else:
                        c[0] = xh + (eo != parity) * (1 + (xh == lxh - 1) * (-lxh))
                else:
                    step = 1 if d == "fwd" else -1
                    c[dim] = (c[dim] + step) % L[dim]
                nb = ((c[3] * Lz + c[2]) * Ly + c[1]) * lxh + c[0]
                M = inp[nb]  # [4][N][m]
                ld = dagger if d == "fwd" else (not dagger)
                sg = -1 if not ld else 1  # sign pattern of the "dagger_flag == 0" branch
                g = dim + 1
                if g == 1:
                    T1 = M[0] + sg * 1j * M[3]; T2 = M[1] + sg * 1j * M[2]
                elif g == 2:
                    T1 = M[0] - sg * M[3]; T2 = M[1] + sg * M[2]
                elif g == 3:
                    T1 = M[0] + sg * 1j * M[2]; T2 = M[1] - sg * 1j * M[3]
                else:
                    T1 = M[0] + sg * M[2]; T2 = M[1] + sg * M[3]
                if d == "fwd":
                    U = gauge[dim, parity, idx]
                else:
                    U = gauge[dim, 1 - parity, nb].conj().T
                R1, R2 = U @ T1, U @ T2
                out[idx, 0] += R1
                out[idx, 1] += R2
                if g == 1:
                    out[idx, 2] += -sg * 1j * R2; out[idx, 3] += -sg * 1j * R1
                elif g == 2:
                    out[idx, 2] += sg * R2; out[idx, 3] += -sg * R1
                elif g == 3:
                    out[idx, 2] += -sg * 1j * R1; out[idx, 3] += sg * 1j * R2
                else:
                    out[idx, 2] += sg * R1; out[idx, 3] += sg * R2
    return out


@pytest.mark.parametrize("dagger", [False, True])
def test_oracle_matches_reference_projector_tables(oracle_lib, dagger):
    O = oracle_lib
    L = (4, 2, 2, 4)
    gauge, psi = _random_problem(L, 3, 2, 6)
    for par in range(2):
        a = F.to_mrhs(psi[:, 1 - par])
        ref = _reference_projector_hop(a, gauge, L, par, dagger)
        assert np.abs(O.hop(a, gauge, L, par, dagger=dagger) - ref).max() < 1e-13


def test_bicgstab_solves_full_system(oracle_lib):
    O = oracle_lib
    L = (4, 4, 4, 4)
    kappa = 0.12
    gauge, psi = _random_problem(L, 3, 3, 7)
    b = np.stack([F.to_mrhs(psi[:, 0]), F.to_mrhs(psi[:, 1])])
    x, it, rr = O.bicgstab(b, gauge, L, kappa, 500, 1e-12)
    assert it > 0 and np.all(rr <= 1e-12)
    xr = np.stack([F.from_mrhs(x[0]), F.from_mrhs(x[1])], axis=1)
    res = O.mat(xr, gauge, L, kappa) - psi
    assert np.linalg.norm(res) / np.linalg.norm(psi) < 1e-11


def test_cgnr_solves_full_system(oracle_lib):
    """The oracle's CGNR (the checker of QCU_SOLVER_CGNR) reaches the same solution as
    the Schur BiCGStab and the FP64 true residual it claims."""
    O = oracle_lib
    L = (4, 4, 4, 4)
    kappa = 0.12
    gauge, psi = _random_problem(L, 3, 3, 7)
    b = np.stack([F.to_mrhs(psi[:, 0]), F.to_mrhs(psi[:, 1])])
    x, it, rr = O.cgnr(b, gauge, L, kappa, 2000, 1e-12)
    assert it > 0 and np.all(rr <= 1e-12)
    xb, _, _ = O.bicgstab(b, gauge, L, kappa, 500, 1e-12)
    assert np.linalg.norm(x - xb) / np.linalg.norm(xb) < 1e-10
    xr = np.stack([F.from_mrhs(x[0]), F.from_mrhs(x[1])], axis=1)
    res = O.mat(xr, gauge, L, kappa) - psi
    assert np.linalg.norm(res) / np.linalg.norm(psi) < 1e-11
    _, it0, _ = O.cgnr(b, gauge, L, kappa, 0, 1e-12)
    assert it0 == -1


def test_bicgstab_zero_iterations_and_zero_source(oracle_lib):
    O = oracle_lib
    L = (4, 2, 2, 2)
    gauge, psi = _random_problem(L, 3, 2, 8)
    b = np.stack([F.to_mrhs(psi[:, 0]), F.to_mrhs(psi[:, 1])])
    x, it, _ = O.bicgstab(b, gauge, L, 0.1, 0, 1e-10)
    assert it == -1


def test_blas_definitions(oracle_lib):
    O = oracle_lib
    rng = np.random.default_rng(9)
    m, n = 5, 37
    a = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
    b = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
    c = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
    s1 = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    s2 = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    s3 = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    assert np.allclose(O.dotc(a, b, m), np.sum(np.conj(a) * b, axis=0))
    assert np.allclose(O.norm(a, m), np.sqrt(np.sum(np.abs(a) ** 2, axis=0)))
    assert np.allclose(O.xsay(a, s1, b, m), a - s1 * b)
    assert np.allclose(O.xpay(a, s1, b, m), a + s1 * b)
    assert np.allclose(O.axpby(s1, a, s2, b, m), s1 * a + s2 * b)
    assert np.allclose(O.axpbypcz(s1, a, s2, b, s3, c, m), s1 * a + s2 * b + s3 * c)


def test_gauge_eo_roundtrip(oracle_lib):
    O = oracle_lib
    L = (4, 2, 6, 2)
    rng = np.random.default_rng(10)
    V = 4 * 2 * 6 * 2
    lex = rng.standard_normal((4, V, 3, 3)) + 1j * rng.standard_normal((4, V, 3, 3))
    eo = O.gauge_to_eo(lex, L)
    assert np.array_equal(O.gauge_from_eo(eo, L), lex)
    # site (x,y,z,t) = (1,0,0,0) is odd: EO index vh + half_index(0,0,0,0)
    vh = V // 2
    assert np.array_equal(eo[2, vh + 0], lex[2, 1])
