"""Backward pass: gradients of a Lennard-Jones loss over the pair list with
respect to positions and cell, against (1) autograd through a reference D
built from the reference's own i, j, S and (2) central FP64 finite
differences with the pair list held fixed (h = 1e-6 A)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS, SIGMA = 1.0, 2.5


def lj(d):
    sr6 = (SIGMA / d) ** 6
    return (4 * EPS * (sr6 * sr6 - sr6)).sum()


def _ref_ijS(oracle, w):
    if oracle.ref_available():
        return oracle.ref_neighbour_list("ijS", w["cell"], w["positions"], w["cutoff"],
                                         w["pbc"])
    return oracle.oracle_neighbour_list("ijS", w["cell"], w["positions"], w["cutoff"],
                                        w["pbc"])


def _grads_ours(w, deterministic=False):
    import torch
    from matscipy_neighbours.autograd import neighbour_list_autograd
    pos = torch.tensor(w["positions"], dtype=torch.float64, device="cuda", requires_grad=True)
    cell = torch.tensor(w["cell"], dtype=torch.float64, device="cuda", requires_grad=True)
    i, j, D, d, S = neighbour_list_autograd(pos, cell, w["pbc"], w["cutoff"],
                                            deterministic=deterministic)
    loss = lj(d)
    loss.backward()
    return (i, j, S), loss.item(), pos.grad.cpu().numpy(), cell.grad.cpu().numpy()


def _grads_ref(w, i, j, S):
    import torch
    pos = torch.tensor(w["positions"], dtype=torch.float64, device="cuda", requires_grad=True)
    cell = torch.tensor(w["cell"], dtype=torch.float64, device="cuda", requires_grad=True)
    ii = torch.as_tensor(i, device="cuda").long()
    jj = torch.as_tensor(j, device="cuda").long()
    SS = torch.as_tensor(S, device="cuda").to(torch.float64)
    D = pos[jj] - pos[ii] + SS @ cell
    loss = lj(torch.linalg.norm(D, dim=1))
    loss.backward()
    return loss.item(), pos.grad.cpu().numpy(), cell.grad.cpu().numpy()


@pytest.mark.parametrize("shape", [(16, 16, 8), (64, 64, 32)])
def test_backward_matches_autograd_through_reference_D(oracle, shape):
    from matscipy_neighbours import _workloads as W
    w = W.diff_lattice(shape=shape)
    (i, j, S), loss, gp, gc = _grads_ours(w)
    ri, rj, rS = _ref_ijS(oracle, w)
    assert np.array_equal(i.cpu().numpy(), ri) and np.array_equal(j.cpu().numpy(), rj)
    assert np.array_equal(S.cpu().numpy(), rS)
    loss_r, gp_r, gc_r = _grads_ref(w, ri, rj, rS)
    assert abs(loss - loss_r) <= 1e-9 * abs(loss_r)
    np.testing.assert_allclose(gp, gp_r, rtol=1e-9, atol=1e-9 * np.abs(gp_r).max())
    np.testing.assert_allclose(gc, gc_r, rtol=1e-9, atol=1e-9 * np.abs(gc_r).max())


def test_backward_central_finite_differences(oracle):
    import torch
    import matscipy_neighbours as m
    from matscipy_neighbours import _workloads as W
    w = W.diff_lattice(shape=(12, 12, 10))
    (i, j, S), loss, gp, gc = _grads_ours(w)
    i, j, S = (t.cpu().numpy() for t in (i, j, S))
    key = oracle.canonical(i, j, S)
    pos0 = torch.tensor(w["positions"], dtype=torch.float64, device="cuda")
    cell0 = torch.tensor(w["cell"], dtype=torch.float64, device="cuda")
    ii = torch.as_tensor(i, device="cuda").long()
    jj = torch.as_tensor(j, device="cuda").long()
    SS = torch.as_tensor(S, device="cuda").to(torch.float64)

    def loss_fixed(pos, cell):
        D = pos[jj] - pos[ii] + SS @ cell
        return lj(torch.linalg.norm(D, dim=1)).item()

    def same_pairs(pos, cell):
        a, b, s = m.neighbour_list("ijS", positions=pos.cpu().numpy(),
                                   cell=cell.cpu().numpy(), pbc=w["pbc"], cutoff=w["cutoff"])
        return np.array_equal(oracle.canonical(a, b, s), key)

    h = 1e-6
    rng = np.random.default_rng(0)
    for flat in rng.choice(pos0.numel(), 12, replace=False):
        a, k = divmod(int(flat), 3)
        p_plus, p_minus = pos0.clone(), pos0.clone()
        p_plus[a, k] += h
        p_minus[a, k] -= h
        assert same_pairs(p_plus, cell0) and same_pairs(p_minus, cell0)
        fd = (loss_fixed(p_plus, cell0) - loss_fixed(p_minus, cell0)) / (2 * h)
        assert abs(fd - gp[a, k]) <= 1e-5 * max(1.0, abs(gp[a, k])), (a, k, fd, gp[a, k])
    for m_ in range(3):
        for k in range(3):
            c_plus, c_minus = cell0.clone(), cell0.clone()
            c_plus[m_, k] += h
            c_minus[m_, k] -= h
            assert same_pairs(pos0, c_plus) and same_pairs(pos0, c_minus)
            fd = (loss_fixed(pos0, c_plus) - loss_fixed(pos0, c_minus)) / (2 * h)
            assert abs(fd - gc[m_, k]) <= 1e-5 * max(1.0, abs(gc[m_, k])), (m_, k, fd, gc[m_, k])


def test_backward_deterministic_is_reproducible():
    from matscipy_neighbours import _workloads as W
    w = W.diff_lattice(shape=(20, 20, 12))
    _, _, gp1, gc1 = _grads_ours(w, deterministic=True)
    _, _, gp2, gc2 = _grads_ours(w, deterministic=True)
    assert np.array_equal(gp1, gp2) and np.array_equal(gc1, gc2)
    _, _, gp3, gc3 = _grads_ours(w, deterministic=False)
    np.testing.assert_allclose(gp3, gp1, rtol=1e-11, atol=1e-11 * np.abs(gp1).max())
    np.testing.assert_allclose(gc3, gc1, rtol=1e-11, atol=1e-11 * np.abs(gc1).max())


def test_backward_distance_vector_only_and_nonperiodic():
    import torch
    from matscipy_neighbours.autograd import neighbour_list_autograd
    rng = np.random.default_rng(3)
    L = 9.0
    cell = np.diag([L, L, L])
    posn = rng.uniform(-1, L + 1, size=(300, 3))  # some atoms outside the box
    for pbc in [(True, True, False), (False, False, False)]:
        pos = torch.tensor(posn, dtype=torch.float64, device="cuda", requires_grad=True)
        c = torch.tensor(cell, dtype=torch.float64, device="cuda", requires_grad=True)
        i, j, D, d, S = neighbour_list_autograd(pos, c, pbc, 2.5)
        wts = torch.linspace(0.1, 1.0, D.shape[0], dtype=torch.float64, device="cuda")
        (D.sum(dim=1) * wts).sum().backward()
        # reference: D = r_j - r_i + (S * pbc) @ cell
        pos2 = torch.tensor(posn, dtype=torch.float64, device="cuda", requires_grad=True)
        c2 = torch.tensor(cell, dtype=torch.float64, device="cuda", requires_grad=True)
        Sp = S.to(torch.float64) * torch.tensor(pbc, dtype=torch.float64, device="cuda")
        D2 = pos2[j.long()] - pos2[i.long()] + Sp @ c2
        torch.testing.assert_close(D2.detach(), D.detach(), rtol=0, atol=1e-12)
        (D2.sum(dim=1) * wts).sum().backward()
        torch.testing.assert_close(pos.grad, pos2.grad, rtol=1e-12, atol=1e-12)
        torch.testing.assert_close(c.grad, c2.grad, rtol=1e-12, atol=1e-10)
