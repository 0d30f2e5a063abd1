"""The hand-written adjoint against (1) autograd through an FP64 PyTorch
restatement of the same discrete dynamics and (2) central finite
differences of the FP64 CPU oracle."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from beads_b200 import workloads
from beads_b200.adjoint import trajectory_observables
from beads_b200.engine import Engine, ReplicaSpec
from tests.adjoint_reference import trajectory

pytestmark = pytest.mark.gpu


def _small(n_replicas=2, n=108, tau=0.05, seed=5):
    specs = workloads.fit_mixture(n_replicas=n_replicas, n=n, density=0.8, tau=tau, seed=seed,
                                  max_neighbors=128)
    for s in specs:
        s.cutoff = 2.2  # rc + skin <= L/2 for the 108-bead boxes
    return specs


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("every", [7, 50, 0])
def test_adjoint_matches_fp64_autograd(every):
    specs = _small()
    steps, rec = 30, 12
    eps0 = torch.tensor(workloads.MIXTURE_EPS, dtype=torch.float64)
    sig0 = torch.tensor(specs[0].sigma, dtype=torch.float64)
    x0 = torch.tensor(np.concatenate([s.positions for s in specs]), dtype=torch.float64)
    v0 = torch.tensor(np.concatenate([s.velocities for s in specs]), dtype=torch.float64)
    rng = np.random.default_rng(0)
    weights = torch.tensor(rng.standard_normal((steps - rec + 1, len(specs), 3)))

    # engine adjoint
    eps = eps0.clone().requires_grad_(True)
    sig = sig0.clone().requires_grad_(True)
    x = x0.clone().requires_grad_(True)
    v = v0.clone().requires_grad_(True)
    with Engine(specs) as eng:
        obs = trajectory_observables(eng, eps, sig, x, v, steps=steps, record_from=rec,
                                     checkpoint_every=every)
        (obs * weights).sum().backward()

    # FP64 autograd reference, replica by replica
    ref_obs, g_eps, g_sig, g_x, g_v = [], torch.zeros(2, 2), torch.zeros(2, 2), [], []
    at = 0
    for r, s in enumerate(specs):
        n = s.n
        e = eps0.clone().requires_grad_(True)
        sg = sig0.clone().requires_grad_(True)
        xr = x0[at:at + n].clone().requires_grad_(True)
        vr = v0[at:at + n].clone().requires_grad_(True)
        box = torch.tensor(np.asarray(s.box_bound[1], np.float64) - s.box_bound[0])
        o = trajectory(xr, vr, torch.tensor(s.masses, dtype=torch.float64),
                       torch.tensor(s.types - 1, dtype=torch.long), box, e, sg, s.cutoff,
                       s.shift, s.dt, steps, rec, thermostat=s.thermostat)
        (o * weights[:, r, :]).sum().backward()
        ref_obs.append(o.detach())
        g_eps = g_eps + e.grad
        g_sig = g_sig + sg.grad
        g_x.append(xr.grad)
        g_v.append(vr.grad)
        at += n
    ref_obs = torch.stack(ref_obs, dim=1)
    assert _rel(obs.detach(), ref_obs) < 1e-5
    assert _rel(eps.grad, g_eps) < 1e-4, (eps.grad, g_eps)
    assert _rel(sig.grad, g_sig) < 1e-4, (sig.grad, g_sig)
    assert _rel(x.grad, torch.cat(g_x)) < 1e-4
    assert _rel(v.grad, torch.cat(g_v)) < 1e-4


def test_adjoint_leaves_end_of_forward_state():
    specs = _small(n_replicas=1)
    eps = torch.tensor(workloads.MIXTURE_EPS, requires_grad=True)
    sig = torch.tensor(specs[0].sigma, requires_grad=True)
    x = torch.tensor(specs[0].positions, dtype=torch.float64, requires_grad=True)
    v = torch.tensor(specs[0].velocities, dtype=torch.float64, requires_grad=True)
    with Engine(specs) as eng:
        obs = trajectory_observables(eng, eps, sig, x, v, steps=20, record_from=10,
                                     checkpoint_every=6)
        after_forward = eng.state()
        obs[:, 0, 0].sum().backward()
        after_backward = eng.state()
        for key in ("positions", "velocities", "images"):
            assert np.array_equal(after_forward[key], after_backward[key]), key
        # and the run continues exactly as it would have
        eng.run(5)


def test_backward_without_forward_is_rejected():
    specs = _small(n_replicas=1)
    with Engine(specs) as eng:
        with pytest.raises(ValueError):
            eng.adjoint_backward(np.zeros((1, 1, 3)))


def _fit_loss(obs, volumes, pe_target, p_target):
    """(<PE> - PE*)^2 + (<P> - P*)^2 per replica, summed; P = (2 KE + W)/(3 V)."""
    pe = obs[:, :, 0].mean(0)
    press = ((2.0 * obs[:, :, 2] + obs[:, :, 1]) / (3.0 * volumes)).mean(0)
    return ((pe - pe_target) ** 2 + (press - p_target) ** 2).sum()


def test_parameter_gradients_match_central_differences():
    """d loss / d(eps_ab, sigma_ab) of the fit loss against central finite
    differences of the FP64 restatement, at relative steps 1e-6 and 1e-3.
    At 1e-6 they agree to 1e-4.  The truncated LJ force jumps at the cutoff,
    so a step of 1e-3 moves pairs across it and the difference quotient then
    differs from the derivative by 0.7% on this run; the FP64 restatement's
    own autograd gradient shows the same gap (6.7e-3), so the bound there is
    3%."""
    specs = _small(seed=9)
    steps, rec = 40, 25
    vols = torch.tensor([float(np.prod(np.asarray(s.box_bound[1], np.float64) - s.box_bound[0]))
                         for s in specs])
    pe_t = torch.tensor([-600.0, -620.0])
    p_t = torch.tensor([1.5, 1.2])
    eps0 = torch.tensor(workloads.MIXTURE_EPS, dtype=torch.float64)
    sig0 = torch.tensor(specs[0].sigma, dtype=torch.float64)
    x0 = torch.tensor(np.concatenate([s.positions for s in specs]), dtype=torch.float64)
    v0 = torch.tensor(np.concatenate([s.velocities for s in specs]), dtype=torch.float64)

    eps = eps0.clone().requires_grad_(True)
    sig = sig0.clone().requires_grad_(True)
    with Engine(specs) as eng:
        obs = trajectory_observables(eng, eps, sig, x0.clone(), v0.clone(), steps=steps,
                                     record_from=rec, checkpoint_every=10)
        _fit_loss(obs, vols, pe_t, p_t).backward()

    def loss_fp64(e, sg):
        rows, at = [], 0
        for s in specs:
            n = s.n
            box = torch.tensor(np.asarray(s.box_bound[1], np.float64) - s.box_bound[0])
            rows.append(trajectory(x0[at:at + n], v0[at:at + n],
                                   torch.tensor(s.masses, dtype=torch.float64),
                                   torch.tensor(s.types - 1, dtype=torch.long), box, e, sg,
                                   s.cutoff, s.shift, s.dt, steps, rec,
                                   thermostat=s.thermostat))
            at += n
        return float(_fit_loss(torch.stack(rows, dim=1), vols, pe_t, p_t))

    for rel, bound in ((1e-6, 1e-4), (1e-3, 3e-2)):
        ours, fd = [], []
        for which, base, grad in (("eps", eps0, eps.grad), ("sig", sig0, sig.grad)):
            for a, b in ((0, 0), (0, 1), (1, 1)):
                h = rel * float(base[a, b])
                plus, minus = base.clone(), base.clone()
                plus[a, b] += h
                minus[a, b] -= h
                if a != b:  # the symmetric table entry moves with it
                    plus[b, a] += h
                    minus[b, a] -= h
                if which == "eps":
                    d = (loss_fp64(plus, sig0) - loss_fp64(minus, sig0)) / (2 * h)
                else:
                    d = (loss_fp64(eps0, plus) - loss_fp64(eps0, minus)) / (2 * h)
                fd.append(d)
                ours.append(float(grad[a, b] + (grad[b, a] if a != b else 0.0)))
        ours, fd = np.array(ours), np.array(fd)
        assert np.linalg.norm(ours - fd) / np.linalg.norm(fd) < bound, (rel, ours, fd)


def test_bonded_adjoint_matches_fp64_autograd():
    """Bead-spring chains (bonds, angles, dihedrals, 1-2/1-3 exclusions):
    gradients w.r.t. positions, velocities, eps, sigma and every harmonic
    parameter against autograd through the FP64 restatement."""
    from oracle import oracle as O
    from tests.test_reference_pin import fixture, tag_ordered

    _, spec = fixture("chains")
    r = tag_ordered(spec)
    n = r.n
    steps, rec = 20, 5
    box = torch.tensor(np.asarray(r.box_bound[1], np.float64) - r.box_bound[0])
    pairs = O.exclusion_pairs(n, r.bonds, r.exclusion_distance)
    excluded = torch.zeros((n, n), dtype=torch.bool)
    for i, j in pairs:
        excluded[i, j] = excluded[j, i] = True
    idx = lambda a, cols: torch.tensor(np.asarray(a, np.int64)[:, :cols] - 1)  # noqa: E731
    top = {"bonds": torch.cat([idx(r.bonds, 2), idx(r.bonds, 3)[:, 2:]], 1),
           "angles": torch.cat([idx(r.angles, 3), idx(r.angles, 4)[:, 3:]], 1),
           "dihedrals": torch.cat([idx(r.dihedrals, 4),
                                   torch.zeros((len(r.dihedrals), 1), dtype=torch.long)], 1)}
    base = {"bond_k": [500.0], "bond_r0": [0.97], "angle_k": [5.0], "angle_theta0": [150.0],
            "dihedral_k": [1.0]}
    rng = np.random.default_rng(3)
    weights = torch.tensor(rng.standard_normal((steps - rec + 1, 1, 3)))
    x0 = torch.tensor(r.positions, dtype=torch.float64)
    v0 = torch.tensor(r.velocities, dtype=torch.float64)

    def leaves():
        out = {k: torch.tensor(v, dtype=torch.float64, requires_grad=True) for k, v in base.items()}
        out["eps"] = torch.tensor(np.asarray(r.epsilon, np.float64), requires_grad=True)
        out["sig"] = torch.tensor(np.asarray(r.sigma, np.float64), requires_grad=True)
        out["x"] = x0.clone().requires_grad_(True)
        out["v"] = v0.clone().requires_grad_(True)
        return out

    ours = leaves()
    with Engine(ReplicaSpec.from_spec(spec)) as eng:
        obs = trajectory_observables(eng, ours["eps"], ours["sig"], ours["x"], ours["v"],
                                     steps=steps, record_from=rec, checkpoint_every=7,
                                     bond_k=ours["bond_k"], bond_r0=ours["bond_r0"],
                                     angle_k=ours["angle_k"], angle_theta0=ours["angle_theta0"],
                                     dihedral_k=ours["dihedral_k"])
        (obs * weights).sum().backward()

    ref = leaves()
    params = {k: ref[k] for k in base}
    params["dihedral_d"] = torch.tensor([1.0], dtype=torch.float64)
    params["dihedral_n"] = torch.tensor([1.0], dtype=torch.float64)
    o = trajectory(ref["x"], ref["v"], torch.tensor(r.masses, dtype=torch.float64),
                   torch.tensor(r.types - 1, dtype=torch.long), box, ref["eps"], ref["sig"],
                   r.cutoff, r.shift, r.dt, steps, rec, thermostat=r.thermostat,
                   excluded=excluded, top=top, params=params)
    (o * weights[:, 0, :]).sum().backward()
    assert _rel(obs.detach()[:, 0, :], o.detach()) < 1e-5
    for key in ("x", "v", "eps", "sig", "bond_k", "bond_r0", "angle_k", "angle_theta0",
                "dihedral_k"):
        assert _rel(ours[key].grad, ref[key].grad) < 1e-4, (key, ours[key].grad, ref[key].grad)


def test_stored_trajectory_gives_the_replayed_gradients_bitwise():
    """checkpoint_every = 0 keeps the forward's own states; replayed segments
    reproduce them bit for bit, so both give the same gradients."""
    specs = _small(n_replicas=1, seed=7)
    grads = []
    for every in (6, 0):
        eps = torch.tensor(workloads.MIXTURE_EPS, requires_grad=True)
        sig = torch.tensor(specs[0].sigma, requires_grad=True)
        x = torch.tensor(specs[0].positions, dtype=torch.float64, requires_grad=True)
        v = torch.tensor(specs[0].velocities, dtype=torch.float64, requires_grad=True)
        with Engine(specs) as eng:
            eng.set_tuning(2, False, 4, True)
            obs = trajectory_observables(eng, eps, sig, x, v, steps=25, record_from=10,
                                         checkpoint_every=every)
            (obs[:, :, 0].sum() + 0.1 * obs[:, :, 1].sum()).backward()
        grads.append((eps.grad.clone(), sig.grad.clone(), x.grad.clone(), v.grad.clone()))
    for a, b in zip(*grads):
        assert torch.equal(a, b)


def test_adjoint_at_fit_scale_matches_fp64_autograd():
    """Two replicas of the 64 x 8192-bead fit workload over 30 steps (the
    loss window's form: weighted PE / virial / KE of the last 20 steps),
    checkpoints every 10 steps, against autograd through the FP64 restatement
    run on the GPU over a fixed pair set with a 2.0 buffer beyond rc (no
    particle moves half of it in 30 steps, so the set holds every pair that
    comes within rc)."""
    from oracle import oracle as O
    from tests.adjoint_reference import trajectory_pairs

    specs = workloads.fit_mixture(n_replicas=2)
    steps, rec, every = 30, 11, 10
    dev = torch.device("cuda", 0)
    eps0 = torch.tensor(workloads.MIXTURE_EPS, dtype=torch.float64)
    sig0 = torch.tensor(specs[0].sigma, dtype=torch.float64)
    x0 = torch.tensor(np.concatenate([s.positions for s in specs]), dtype=torch.float64)
    v0 = torch.tensor(np.concatenate([s.velocities for s in specs]), dtype=torch.float64)
    rng = np.random.default_rng(1)
    weights = torch.tensor(rng.standard_normal((steps - rec + 1, len(specs), 3)))
    weights[:, :, 0] /= 8192.0  # PE and virial are extensive: comparable terms
    weights[:, :, 1] /= 8192.0

    eps = eps0.clone().requires_grad_(True)
    sig = sig0.clone().requires_grad_(True)
    x = x0.clone().requires_grad_(True)
    v = v0.clone().requires_grad_(True)
    with Engine(specs) as eng:
        obs = trajectory_observables(eng, eps, sig, x, v, steps=steps, record_from=rec,
                                     checkpoint_every=every)
        (obs * weights).sum().backward()

    buffer = 2.0
    g_eps, g_sig, g_x, g_v, ref_obs = 0.0, 0.0, [], [], []
    at = 0
    for r, s in enumerate(specs):
        n = s.n
        counts, partners = O.neighbors(s.positions, s.box_bound, s.cutoff, buffer, cap=512)
        rows = np.repeat(np.arange(n), counts)
        cols = np.concatenate([partners[i, :counts[i]] for i in range(n)])
        keep = rows < cols
        pi = torch.tensor(rows[keep], device=dev)
        pj = torch.tensor(cols[keep].astype(np.int64), device=dev)
        e = eps0.to(dev).clone().requires_grad_(True)
        sg = sig0.to(dev).clone().requires_grad_(True)
        xr = x0[at:at + n].to(dev).clone().requires_grad_(True)
        vr = v0[at:at + n].to(dev).clone().requires_grad_(True)
        box = torch.tensor(np.asarray(s.box_bound[1], np.float64) - s.box_bound[0], device=dev)
        o, moved = trajectory_pairs(xr, vr, torch.tensor(s.masses, dtype=torch.float64,
                                                         device=dev),
                                    torch.tensor(s.types - 1, dtype=torch.long, device=dev),
                                    box, e, sg, s.cutoff, s.shift, s.dt, steps, rec, pi, pj,
                                    thermostat=s.thermostat)
        assert moved < 0.5 * buffer, moved
        (o * weights[:, r, :].to(dev)).sum().backward()
        ref_obs.append(o.detach().cpu())
        g_eps = g_eps + e.grad.cpu()
        g_sig = g_sig + sg.grad.cpu()
        g_x.append(xr.grad.cpu())
        g_v.append(vr.grad.cpu())
        at += n
    ref_obs = torch.stack(ref_obs, dim=1)
    assert _rel(obs.detach(), ref_obs) < 1e-5
    assert _rel(eps.grad, g_eps) < 1e-4, (eps.grad, g_eps)
    assert _rel(sig.grad, g_sig) < 1e-4, (sig.grad, g_sig)
    assert _rel(x.grad, torch.cat(g_x)) < 1e-4
    assert _rel(v.grad, torch.cat(g_v)) < 1e-4
