"""The differentiable form (protomoladdon_b200.autograd) on the GPU against
FP64 central finite differences of the CPU oracle (h = 1e-4) and against
ProtoMol's own analytic Hessian (oracle/ref_hessian.cpp).

Tolerances (written here, checked below):
* Hessian-vector products (FP64 kernel): relative to |Hv|, <= 1e-10 against
  the reference's analytic Hessian, <= 1e-6 against finite differences of
  the oracle's forces (the finite-difference error is ~1e-9).
* parameter gradients (FP64 kernel): relative <= 1e-6 against finite
  differences of the oracle's energy.
* dE/dx through the mixed force kernel: RMS relative <= 1e-5; through the
  FP64 kernel <= 1e-12.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from protomoladdon_b200 import water
from protomoladdon_b200.autograd import NonbondedEnergy, SQRTCOULOMBCONSTANT, lj_table
from protomoladdon_b200.force import PeriodicTopology

from .conftest import load_fixture

pytestmark = pytest.mark.gpu

H = 1e-4


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def oracle_forces(s, pos, q=None, lj=None):
    d = dict(s)
    if q is not None:
        d["qscaled"] = q
    if lj is not None:
        d["lj"] = lj
    f, e, _, _ = O.restate_eval(d, pos, virial_mode=0)
    return f, float(e.sum())


@pytest.fixture(scope="module")
def small():
    return water.small_648()


@pytest.fixture(scope="module")
def ions():
    return water.water_box(6, rc=8.0, ron=7.0, seed=21, ion_fraction=0.1)


def make(s, precision="fp64"):
    m = NonbondedEnergy.from_system(s, precision=precision)
    q, t = m.initial_params()
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    return m, pos, q, t


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_energy_and_position_gradient(small, precision, tol):
    m, pos, q, t = make(small, precision)
    pos.requires_grad_(True)
    E = m.energy(pos, q, t)
    (g,) = torch.autograd.grad(E, pos)
    fo, eo = oracle_forces(small, small["pos"])
    m.close()
    assert abs(E.item() - eo) <= (1e-12 if precision == "fp64" else 2e-3) * max(1.0, abs(eo))
    assert rel(-g.cpu().numpy(), fo) <= tol


@pytest.mark.parametrize("fx", ["small", "ions"])
def test_hvp_against_reference_hessian_and_fd(fx, request):
    """32 seeded unit directions by double backward, against the reference's
    analytic Hessian; 4 of them against finite differences too."""
    s = request.getfixturevalue(fx)
    m, pos, q, t = make(s)
    R = O.RefForce(s)
    Hm = R.hessian(s["pos"])
    R.close()
    rng = np.random.default_rng(2024)
    pos.requires_grad_(True)
    E = m.energy(pos, q, t)
    (g,) = torch.autograd.grad(E, pos, create_graph=True)
    for k in range(32):
        v = rng.standard_normal(s["pos"].shape)
        v /= np.linalg.norm(v)
        vt = torch.tensor(v, dtype=torch.float64, device="cuda")
        (hv,) = torch.autograd.grad(g, pos, grad_outputs=vt, retain_graph=True)
        hv = hv.cpu().numpy()
        ref = (Hm @ v.reshape(-1)).reshape(-1, 3)
        assert rel(hv, ref) <= 1e-10, (k, rel(hv, ref))
        if k < 4:
            fp, _ = oracle_forces(s, s["pos"] + H * v)
            fm, _ = oracle_forces(s, s["pos"] - H * v)
            assert rel(hv, -(fp - fm) / (2 * H)) <= 1e-6
    m.close()


def test_charge_and_type_gradients_against_fd(ions):
    """dE/dq (atoms of every type) and dE/dsigma, dE/depsilon per type through
    lj_table, against central differences of the oracle's energy."""
    s = ions
    m, pos, q0, _ = make(s)
    sig = torch.tensor([3.1507, 0.0, 2.43, 4.04], dtype=torch.float64, device="cuda",
                       requires_grad=True)
    eps = torch.tensor([0.1521, 0.0, 0.047, 0.15], dtype=torch.float64, device="cuda",
                       requires_grad=True)
    q = q0.clone().requires_grad_(True)
    table = lj_table(sig, eps)
    np.testing.assert_allclose(table.detach().cpu().numpy(), s["lj"], rtol=1e-12, atol=0)
    E = m.energy(pos, q, table)
    gq, gs, ge = torch.autograd.grad(E, (q, sig, eps))
    m.close()
    qh = np.asarray(s["qscaled"], float)
    for i in [0, 1, 2] + [int(k) for k in np.nonzero(s["type"] >= 2)[0][:4]]:
        dq = np.zeros_like(qh)
        dq[i] = H
        _, ep = oracle_forces(s, s["pos"], q=qh + dq)
        _, em = oracle_forces(s, s["pos"], q=qh - dq)
        fd = (ep - em) / (2 * H)
        assert abs(gq[i].item() - fd) <= 1e-6 * max(abs(fd), 1.0), (i, gq[i].item(), fd)

    def energy_with(sg, ep_):
        tb = lj_table(torch.tensor(sg, dtype=torch.float64),
                      torch.tensor(ep_, dtype=torch.float64)).numpy()
        return oracle_forces(s, s["pos"], lj=tb)[1]

    s0 = sig.detach().cpu().numpy()
    e0 = eps.detach().cpu().numpy()
    for a in (0, 2, 3):
        for base, grad in ((s0, gs), (e0, ge)):
            p = base.copy()
            p[a] += H * base[a]
            up = energy_with(p, e0) if base is s0 else energy_with(s0, p)
            p[a] -= 2 * H * base[a]
            dn = energy_with(p, e0) if base is s0 else energy_with(s0, p)
            fd = (up - dn) / (2 * H * base[a])
            assert abs(grad[a].item() - fd) <= 1e-6 * max(abs(fd), 1e-3), (a, grad[a].item(), fd)


def test_force_matching_loss_gradient(small):
    """d/dtheta of sum |F(theta) - F_target|^2 (the mixed second derivatives)
    against central differences of the same loss from the oracle's forces;
    F_target from parameters with 5% seeded Gaussian perturbations."""
    s = small
    m, pos, q0, _ = make(s)
    rng = np.random.default_rng(7)
    sig0 = np.array([3.1507, 0.0])
    eps0 = np.array([0.1521, 0.0])
    sig_t = sig0 * (1 + 0.05 * rng.standard_normal(2))
    eps_t = eps0 * (1 + 0.05 * rng.standard_normal(2))
    qt = np.asarray(s["qscaled"]) * (1 + 0.05 * rng.standard_normal())  # one overall factor
    tt = lj_table(torch.tensor(sig_t), torch.tensor(eps_t)).numpy()
    F_t, _ = oracle_forces(s, s["pos"], q=qt, lj=tt)
    sig = torch.tensor(sig0, device="cuda", requires_grad=True)
    eps = torch.tensor(eps0, device="cuda", requires_grad=True)
    q = q0.clone().requires_grad_(True)
    F = m.forces(pos, q, lj_table(sig, eps))
    Ft = torch.tensor(F_t, device="cuda")
    loss = ((F - Ft) ** 2).sum()
    gs, ge, gq = torch.autograd.grad(loss, (sig, eps, q))
    m.close()

    def loss_with(sg, ep_, qq):
        tb = lj_table(torch.tensor(sg), torch.tensor(ep_)).numpy()
        f, _ = oracle_forces(s, s["pos"], q=qq, lj=tb)
        return float(((f - F_t) ** 2).sum())

    qh = np.asarray(s["qscaled"], float)

    def richardson(f, x0, h):
        # central differences at h and h/2, extrapolated (error O(h^4)): the
        # loss varies like sigma^24, too sharply for a plain h = 1e-4 step
        d1 = (f(x0 + h) - f(x0 - h)) / (2 * h)
        d2 = (f(x0 + h / 2) - f(x0 - h / 2)) / h
        return (4 * d2 - d1) / 3

    fd_s = richardson(lambda x: loss_with(np.array([x, 0.0]), eps0, qh), sig0[0], H * sig0[0])
    fd_e = richardson(lambda x: loss_with(sig0, np.array([x, 0.0]), qh), eps0[0], H * eps0[0])
    assert abs(gs[0].item() - fd_s) <= 1e-5 * abs(fd_s), (gs[0].item(), fd_s)
    assert abs(ge[0].item() - fd_e) <= 1e-5 * abs(fd_e), (ge[0].item(), fd_e)
    for i in (0, 1, 333):
        dq = np.zeros_like(qh)
        dq[i] = H
        fd = (loss_with(sig0, eps0, qh + dq) - loss_with(sig0, eps0, qh - dq)) / (2 * H)
        assert abs(gq[i].item() - fd) <= 1e-5 * max(abs(fd), 1e-3), (i, gq[i].item(), fd)


def test_medium_box_hvp_and_charge_gradient_against_fd():
    s = water.medium_41k()
    m, pos, q, t = make(s)
    rng = np.random.default_rng(5)
    v = rng.standard_normal(s["pos"].shape)
    v /= np.linalg.norm(v)
    hv = torch.empty_like(pos)
    vt = torch.tensor(v, device="cuda")
    m.force.hvp_device(m.topo, pos.data_ptr(), vt.data_ptr(), hv.data_ptr())
    dq = torch.empty_like(q)
    dt = torch.empty_like(t)
    m.force.param_grad_device(m.topo, pos.data_ptr(), dq.data_ptr(), dt.data_ptr())
    torch.cuda.synchronize()
    m.close()
    fp, _ = oracle_forces(s, s["pos"] + H * v)
    fm, _ = oracle_forces(s, s["pos"] - H * v)
    assert rel(hv.cpu().numpy(), -(fp - fm) / (2 * H)) <= 1e-6
    qh = np.asarray(s["qscaled"], float)
    dd = np.zeros_like(qh)
    dd[100] = H
    _, ep = oracle_forces(s, s["pos"], q=qh + dd)
    _, em = oracle_forces(s, s["pos"], q=qh - dd)
    fd = (ep - em) / (2 * H)
    assert abs(dq[100].item() - fd) <= 1e-6 * abs(fd)


@pytest.fixture(scope="module")
def medium():
    return water.medium_41k()


@pytest.mark.parametrize("fx", ["small", "ions", "medium"])
def test_hvp_half_shell_kernel(fx, request):
    """A plain Hessian-vector product (the half-shell kernel, each pair once,
    fixed-point sums) against the same product asked with dE/dq (the
    kernel's parameter instance): relative <= 1e-12; two plain products
    bit-identical."""
    s = request.getfixturevalue(fx)
    m, pos, q, t = make(s)
    rng = np.random.default_rng(11)
    v = rng.standard_normal(s["pos"].shape)
    vt = torch.tensor(v / np.linalg.norm(v), device="cuda")
    h1, h2, hf = (torch.empty_like(pos) for _ in range(3))
    m.force.hvp_device(m.topo, pos.data_ptr(), vt.data_ptr(), h1.data_ptr())
    m.force.hvp_device(m.topo, pos.data_ptr(), vt.data_ptr(), h2.data_ptr())
    dq = torch.empty_like(q)
    m.force.hvp_device(m.topo, pos.data_ptr(), vt.data_ptr(), hf.data_ptr(), dq.data_ptr())
    torch.cuda.synchronize()
    m.force.sync()
    m.close()
    assert torch.equal(h1, h2)
    assert rel(h1.cpu().numpy(), hf.cpu().numpy()) <= 1e-12


def test_vacuum_hvp_and_charge_gradient():
    """Vacuum boundaries (the water droplet of the reference's vacuum
    fixture): H w and dE/dq against central differences of the reference's
    own vacuum cutoff force and energy (oracle/_ref), h = 1e-4."""
    d = dict(load_fixture("vacuum_ref.npz"))
    topo = PeriodicTopology.from_dict(d)
    topo.domain = (d["pos"].min(0) - 1.0, d["pos"].max(0) + 1.0)
    m = NonbondedEnergy(topo, d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"], precision="fp64")
    q, _ = m.initial_params()
    pos = torch.tensor(d["pos"], dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(9)
    v = rng.standard_normal(d["pos"].shape)
    v /= np.linalg.norm(v)
    vt = torch.tensor(v, device="cuda")
    hv = torch.empty_like(pos)
    m.force.hvp_device(m.topo, pos.data_ptr(), vt.data_ptr(), hv.data_ptr())
    dq = torch.empty_like(q)
    dt = torch.empty(len(d["lj"]) ** 2 * 4, dtype=torch.float64, device="cuda")
    m.force.param_grad_device(m.topo, pos.data_ptr(), dq.data_ptr(), dt.data_ptr())
    torch.cuda.synchronize()
    m.force.sync()
    m.close()
    fp = O.ref_vacuum_eval(d, d["pos"] + H * v, virial_mode=0)[0]
    fm = O.ref_vacuum_eval(d, d["pos"] - H * v, virial_mode=0)[0]
    assert rel(hv.cpu().numpy(), -(fp - fm) / (2 * H)) <= 1e-6
    qh = np.asarray(d["qscaled"], float)
    for i in (0, 1, 100):
        dd = np.zeros_like(qh)
        dd[i] = H
        ep = O.ref_vacuum_eval(dict(d, qscaled=qh + dd), d["pos"], virial_mode=0)[1].sum()
        em = O.ref_vacuum_eval(dict(d, qscaled=qh - dd), d["pos"], virial_mode=0)[1].sum()
        fd = (ep - em) / (2 * H)
        assert abs(dq[i].item() - fd) <= 1e-6 * max(abs(fd), 1.0), (i, dq[i].item(), fd)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_parameter_update(small, precision):
    """pmb200_update_params_device against pmb200_update_params (host): the
    same forces and energies bit for bit, again after a box change (which
    rebuilds the FP32 table from the device-updated one); a non-finite
    charge is reported by the next sync, and the context stays usable."""
    from protomoladdon_b200._lib import PmbError
    from protomoladdon_b200.force import NonbondedCutoffB200SystemForce, ScalarStructure
    s = small
    q2 = np.asarray(s["qscaled"]) * 1.05
    lj2 = np.asarray(s["lj"]) * np.array([1.1, 0.9, 1.2, 0.8])
    out = []
    for mode in ("host", "device"):
        topo = PeriodicTopology.from_dict(s)
        f = NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"],
                                           precision=precision)
        if mode == "host":
            f.update_params(topo, q2, lj2)
        else:
            qd = torch.tensor(q2, device="cuda")
            td = torch.tensor(lj2, device="cuda")
            torch.cuda.synchronize()
            f.update_params_device(topo, qd.data_ptr(), td.data_ptr())  # the context's stream
        res = []
        e0 = topo.e.copy()
        for scale in (1.0, 1.01):
            topo.e = np.ascontiguousarray(e0 * scale)
            F = np.zeros_like(s["pos"])
            E = ScalarStructure()
            f.evaluate(topo, s["pos"], F, E)
            res.append((F, E[0], E[1]))
        if mode == "device":
            bad = qd.clone()
            bad[5] = float("nan")
            f.update_params_device(topo, bad.data_ptr(), None)
            with pytest.raises(PmbError):
                f.sync()
            f.update_params_device(topo, qd.data_ptr(), None)
            F = np.zeros_like(s["pos"])
            E = ScalarStructure()
            f.evaluate(topo, s["pos"], F, E)
            res.append((F, E[0], E[1]))
        f.close()
        out.append(res)
    host, dev = out
    for (Fh, ch, lh), (Fd, cd, ld) in zip(host, dev):
        assert np.array_equal(Fh, Fd) and ch == cd and lh == ld
    assert np.array_equal(dev[2][0], dev[1][0]) and dev[2][1] == dev[1][1]


def split_types(d, extra=((0, 4), (1, 5))):
    """The same atoms over more LJ types: every other atom of type a moves to
    a new type b carrying a's parameters (the table's rows and columns
    copied), so the energy, the forces, dE/dq and H w are unchanged and the
    table derivative folds back onto the original entries.  Returns the
    system and each type's original type."""
    typ = np.asarray(d["type"]).copy()
    nt = d["lj"].shape[0]
    orig = np.array(list(range(nt)) + [a for a, _ in extra])
    for a, b in extra:
        typ[np.flatnonzero(typ == a)[::2]] = b
    out = dict(d)
    out["type"] = typ.astype(np.int32)
    out["lj"] = d["lj"][np.ix_(orig, orig)].copy()
    return out, orig


@pytest.mark.parametrize("mode", ["params", "vjp"])
def test_derivative_kernels_agree_across_type_counts(ions, mode):
    """The ion box over its four LJ types (parameter derivatives by the
    half-shell kernel, each pair once) against the same box over six types
    (the full-shell kernel, each pair from both atoms): dE/dq, the table
    derivative folded back onto the four types and, in VJP mode, H w, all
    within 1e-12 relative."""
    s6, orig = split_types(ions)
    assert len(orig) == 6 and (np.bincount(s6["type"], minlength=6) > 0).all()
    res = []
    for s in (ions, s6):
        m, pos, q, t = make(s)
        dq = torch.empty_like(q)
        dt = torch.empty(t.shape, dtype=torch.float64, device="cuda")
        hv = torch.zeros_like(pos)
        if mode == "params":
            m.force.param_grad_device(m.topo, pos.data_ptr(), dq.data_ptr(), dt.data_ptr())
        else:
            v = np.random.default_rng(3).standard_normal(s["pos"].shape)
            vt = torch.tensor(v / np.linalg.norm(v), device="cuda")
            m.force.hvp_device(m.topo, pos.data_ptr(), vt.data_ptr(), hv.data_ptr(),
                               dq.data_ptr(), dt.data_ptr())
        torch.cuda.synchronize()
        m.force.sync()
        m.close()
        res.append((dq.cpu().numpy(), dt.cpu().numpy().reshape(len(s["lj"]), -1, 4),
                    hv.cpu().numpy()))
    (dq4, dt4, hv4), (dq6, dt6, hv6) = res
    folded = np.zeros_like(dt4)
    for a in range(6):
        for b in range(6):
            folded[orig[a], orig[b]] += dt6[a, b]
    assert rel(dq4, dq6) <= 1e-12
    assert rel(dt4, folded) <= 1e-12
    if mode == "vjp":
        assert rel(hv4, hv6) <= 1e-12


def test_charge_units_constant():
    assert SQRTCOULOMBCONSTANT ** 2 == pytest.approx(332.0636, rel=1e-6)
