"""Energy and adjoint (p3mg_energy / p3mg_backward; no reference
counterpart): every gradient against central finite differences of the
energy in FP64 (h = 1e-4), the energy against an independent Ewald sum,
FP32 against FP64, and a test-only torch.autograd.Function over the same
C ABI."""
import numpy as np
import pytest

import oracle as O
import p3mg

pytestmark = pytest.mark.gpu
H = 1e-4


def energy_at(method, mesh, cao, mc, alpha, rcut, x, y, z, q, L, precision=p3mg.FP64):
    with p3mg.Context(method, mesh, cao, mc, precision) as ctx:
        ctx.set_system(x, y, z, q, L)
        ctx.influence(alpha)
        return ctx.energy(rcut)["total"]


def adjoint_at(method, mesh, cao, mc, alpha, rcut, x, y, z, q, L, precision=p3mg.FP64):
    with p3mg.Context(method, mesh, cao, mc, precision) as ctx:
        ctx.set_system(x, y, z, q, L)
        ctx.influence(alpha)
        return ctx.backward(rcut)


def fd_check(method, mesh, cao, mc, alpha, rcut, x, y, z, q, L, coords, tol):
    g = adjoint_at(method, mesh, cao, mc, alpha, rcut, x, y, z, q, L)
    E = lambda *a, **k: energy_at(method, mesh, cao, mc, *a, **k)  # noqa: E731
    pos = [x, y, z]
    num, ana = [], []
    for i in coords:
        for d in range(3):
            p = [v.copy() for v in pos]
            p[d][i] += H
            ep = E(alpha, rcut, *p, q, L)
            p[d][i] -= 2 * H
            em = E(alpha, rcut, *p, q, L)
            num.append((ep - em) / (2 * H))
            ana.append(g["dx"][d][i])
        qp, qm = q.copy(), q.copy()
        qp[i] += H
        qm[i] -= H
        num.append((E(alpha, rcut, x, y, z, qp, L) - E(alpha, rcut, x, y, z, qm, L)) / (2 * H))
        ana.append(g["dq"][i])
    num, ana = np.array(num), np.array(ana)
    assert np.linalg.norm(ana - num) <= tol * np.linalg.norm(num), (ana, num)
    # alpha
    da = (E(alpha + H, rcut, x, y, z, q, L) - E(alpha - H, rcut, x, y, z, q, L)) / (2 * H)
    assert abs(g["dalpha"] - da) <= tol * max(abs(da), 1e-3 * abs(g["energy"]["total"]))
    # box length at fixed fractional coordinates
    sp, sm = (L + H) / L, (L - H) / L
    dl = (E(alpha, rcut, x * sp, y * sp, z * sp, q, L + H) - E(alpha, rcut, x * sm, y * sm, z * sm, q, L - H)) / (2 * H)
    assert abs(g["dL"] - dl) <= tol * abs(dl)
    return g


def test_adjoint_fd_separated_dipoles_method2(gpu):
    # the differentiation configuration on a 32-particle copy: 16 dipoles,
    # box 46.4, mesh 64, cao 5, rcut 3, alpha 1
    x, y, z, q = p3mg.generate_system(3, 32, 46.4, seed=61)
    fd_check(2, 64, 5, 1, 1.0, 3.0, x, y, z, q, 46.4, range(32), 1e-6)


@pytest.mark.parametrize("method", [0, 1, 3, 6, 7])
def test_adjoint_fd_all_methods(gpu, method):
    x, y, z, q = p3mg.generate_system(0, 40, 6.0, seed=62 + method)
    fd_check(method, 16, 5, 1, 1.1, 2.4, x, y, z, q, 6.0, range(0, 40, 3), 1e-6)


def test_adjoint_fd_charged_system(gpu):
    # net charge: the neutralising term and its derivatives
    x, y, z, q = p3mg.generate_system(0, 30, 6.0, seed=70)
    q[:5] = 1.0
    fd_check(1, 16, 4, 1, 1.0, 2.4, x, y, z, q, 6.0, range(0, 30, 4), 1e-6)


def ewald_energy(x, y, z, q, L, alpha, kmax):
    # independent reference: plain Ewald with full minimum-image real space
    # (rcut = L/2) and the k-space sum to |n| <= kmax
    pos = np.stack([x, y, z], 1)
    d = pos[:, None, :] - pos[None, :, :]
    d -= L * np.round(d / L)
    r = np.sqrt((d ** 2).sum(-1))
    np.fill_diagonal(r, np.inf)
    from scipy.special import erfc
    er = 0.5 * np.sum(np.outer(q, q) * np.where(r <= L / 2, erfc(alpha * r) / r, 0.0))
    ns = np.arange(-kmax, kmax + 1)
    nx, ny, nz = np.meshgrid(ns, ns, ns, indexing="ij")
    n = np.stack([nx.ravel(), ny.ravel(), nz.ravel()], 1)
    n2 = (n ** 2).sum(1)
    keep = (n2 > 0) & (n2 <= kmax * kmax)
    n, n2 = n[keep], n2[keep]
    S = np.exp(-2j * np.pi * (n @ pos.T) / L) @ q
    ek = np.sum(np.exp(-(np.pi ** 2) * n2 / (alpha * L) ** 2) / n2 * np.abs(S) ** 2) / (2 * np.pi * L)
    return er + ek - alpha / np.sqrt(np.pi) * np.sum(q * q) - np.pi * q.sum() ** 2 / (2 * alpha ** 2 * L ** 3)


@pytest.mark.parametrize("method", [0, 1, 2, 3, 6, 7])
def test_energy_matches_ewald(gpu, method):
    L, alpha = 8.0, 1.2
    x, y, z, q = p3mg.generate_system(0, 200, L, seed=71)
    e_ref = ewald_energy(x, y, z, q, L, 0.9, 14)  # converged Ewald: any alpha
    with p3mg.Context(method, 32, 7, 2) as ctx:
        ctx.set_system(x, y, z, q, L)
        ctx.influence(alpha)
        e = ctx.energy(3.9)
    scale = abs(e["kspace"]) + abs(e["realspace"]) + abs(e["self"])
    assert abs(e["total"] - e_ref) <= 2e-4 * scale, (e, e_ref)


def test_fp32_adjoint_matches_fp64(gpu):
    x, y, z, q = p3mg.generate_system(3, 20000, 21.5, seed=72)
    g64 = adjoint_at(2, 32, 5, 1, 1.0, 3.0, x, y, z, q, 21.5)
    g32 = adjoint_at(2, 32, 5, 1, 1.0, 3.0, x, y, z, q, 21.5, precision=p3mg.FP32_MIXED)
    assert abs(g32["energy"]["total"] - g64["energy"]["total"]) <= 1e-5 * abs(g64["energy"]["total"])
    assert O.rel_rms(g32["dx"].ravel(), g64["dx"].ravel()) <= 1e-4
    assert O.rel_rms(g32["dq"], g64["dq"]) <= 1e-4
    assert abs(g32["dalpha"] - g64["dalpha"]) <= 1e-4 * abs(g64["energy"]["total"])


def test_ad_gradient_is_minus_ad_force(gpu):
    # method 3 (ad, interlaced, no self-force correction): the force pipeline
    # differs from -dE/dx only by the 2^-17 binning of the weights
    x, y, z, q = p3mg.generate_system(0, 2000, 13.0, seed=73)
    with p3mg.Context(3, 32, 6, 1) as ctx:
        ctx.set_system(x, y, z, q, 13.0)
        ctx.influence(1.0)
        f = ctx.calculate_forces(3.2)["f"]
        g = ctx.backward(3.2)
    assert O.rel_rms((-g["dx"]).ravel(), f.ravel()) <= 1e-4


def test_torch_autograd_wrapper(gpu):
    torch = pytest.importorskip("torch")

    class P3MEnergy(torch.autograd.Function):
        """Test-only: the P3M energy as a torch function of (x, q, L, alpha)
        with its backward from p3mg_backward."""

        @staticmethod
        def forward(fctx, pos, q, L, alpha, method, mesh, cao, rcut):
            p = pos.detach().cpu().numpy().astype(np.float64)
            qq = q.detach().cpu().numpy().astype(np.float64)
            with p3mg.Context(method, mesh, cao, 1) as c:
                c.set_system(p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), qq, float(L))
                c.influence(float(alpha))
                g = c.backward(rcut)
            fctx.save_for_backward(torch.tensor(g["dx"].T.copy()), torch.tensor(g["dq"]),
                                   torch.tensor(g["dL"]), torch.tensor(g["dalpha"]))
            return torch.tensor(g["energy"]["total"], dtype=torch.float64)

        @staticmethod
        def backward(fctx, ge):
            dx, dq, dl, da = fctx.saved_tensors
            return ge * dx, ge * dq, ge * dl, ge * da, None, None, None, None

    x, y, z, q = p3mg.generate_system(3, 32, 46.4, seed=61)
    pos = torch.tensor(np.stack([x, y, z], 1), requires_grad=True)
    qt = torch.tensor(q, requires_grad=True)
    Lt = torch.tensor(46.4, dtype=torch.float64, requires_grad=True)
    at = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    E = P3MEnergy.apply(pos, qt, Lt, at, 2, 64, 5, 3.0)
    (3.0 * E).backward()
    # chain rule through the wrapper, and the gradient against finite differences
    i, d = 5, 1
    p = [x.copy(), y.copy(), z.copy()]
    p[d][i] += H
    ep = energy_at(2, 64, 5, 1, 1.0, 3.0, *p, q, 46.4)
    p[d][i] -= 2 * H
    em = energy_at(2, 64, 5, 1, 1.0, 3.0, *p, q, 46.4)
    assert abs(pos.grad[i, d].item() - 3.0 * (ep - em) / (2 * H)) <= 1e-6 * abs(3.0 * (ep - em) / (2 * H))
    assert qt.grad is not None and Lt.grad is not None and at.grad is not None


@pytest.mark.parametrize("precision", [p3mg.FP64, p3mg.FP32_MIXED])
def test_backward_device_matches_host(gpu, precision):
    # p3mg_backward_device leaves the gradients on the GPU: the same numbers
    # as p3mg_backward's host arrays, two calls in a row
    import ctypes
    x, y, z, q = p3mg.generate_system(3, 4000, 21.5, seed=17)
    with p3mg.Context(1, 32, 5, 1, precision) as ctx:
        ctx.set_system(x, y, z, q, 21.5)
        ctx.influence(1.0)
        h = ctx.backward(3.0, grad_E=2.0)
        for _ in range(2):
            d = ctx.backward_device(3.0, grad_E=2.0)
            n = len(x)
            gx, gq = np.zeros(3 * n), np.zeros(n)
            cudart = ctypes.CDLL("libcudart.so")
            cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
            assert cudart.cudaMemcpy(gx.ctypes.data, d["dx_ptr"], gx.nbytes, 2) == 0
            assert cudart.cudaMemcpy(gq.ctypes.data, d["dq_ptr"], gq.nbytes, 2) == 0
            # the mesh sums take global atomics across bricks: equal up to
            # the rounding of their order
            tol = 1e-12 if precision == p3mg.FP64 else 1e-6
            assert O.rel_rms(gx.reshape(3, n), h["dx"]) <= tol
            assert O.rel_rms(gq, h["dq"]) <= tol
            assert abs(d["dalpha"] - h["dalpha"]) <= tol * abs(h["energy"]["total"])
            assert abs(d["energy"]["total"] - h["energy"]["total"]) <= tol * abs(h["energy"]["total"])
