"""The differentiable unrolled TGV solve on the GPU (unround.unrolled): its forward map against
the FP64 CPU reference (oracle/unrolled_torch.py, itself pinned to the reference's C++ solver),
the adjoint's gradients with respect to alpha0, alpha1, tau and sigma against the reference's
autograd gradients and against central finite differences of the device's own forward map
(h = 1e-3), and the gradients' independence of the checkpoints' spacing. The device computes in
binary32: forward within rel L2 1e-5 of the reference, gradients within 2e-3 (relative)."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

OPTIONS = ["--method", "tgv", "--alpha1", "1", "--alpha0", "2"]


def _case(iterations=20, every=6, rows=64, columns=72, pictures=2):
    from unround import synthetic
    from unround.unrolled import UnrolledProblem

    made = [synthetic.grey(rows, columns, quality=30, seed=10 + s, noise=2) for s in range(pictures)]
    problem = UnrolledProblem([m.image for m in made], OPTIONS, iterations=iterations, checkpoint_every=every)
    clean = torch.tensor(np.stack([m.samples for m in made]), dtype=torch.float32, device="cuda")
    base = [np.linspace(2.0, 1.5, pictures), np.linspace(1.0, 0.8, pictures),
            problem.tau * np.linspace(1.0, 0.9, pictures), problem.sigma * np.linspace(1.0, 1.1, pictures)]
    return problem, clean, base


def _device_loss_and_grads(problem, clean, base):
    from unround.unrolled import unrolled_tgv

    leaves = [torch.tensor(b, dtype=torch.float32, device="cuda", requires_grad=True) for b in base]
    out = unrolled_tgv(problem, *leaves)
    loss = torch.mean((out.double() - clean.double()) ** 2)
    loss.backward()
    return out.detach(), loss.item(), [leaf.grad.double().cpu().numpy() for leaf in leaves]


def _reference_grads(problem, clean, base):
    from oracle.unrolled_torch import Reference

    ref = Reference(problem)
    leaves = [torch.tensor(b, dtype=torch.float64, requires_grad=True) for b in base]
    out = ref.run(*leaves, problem.iterations)
    loss = torch.mean((out - clean.double().cpu()) ** 2)
    loss.backward()
    return out.detach().numpy(), [leaf.grad.numpy() for leaf in leaves]


def test_forward_and_gradients_against_the_reference():
    problem, clean, base = _case()
    out, _, grads = _device_loss_and_grads(problem, clean, base)
    ref_out, ref_grads = _reference_grads(problem, clean, base)
    got = out.double().cpu().numpy()
    assert np.linalg.norm(got - ref_out) / np.linalg.norm(ref_out) <= 1e-5
    assert np.abs(got - ref_out).max() <= 1e-3
    for k, (g, r) in enumerate(zip(grads, ref_grads)):
        scale = np.abs(r).max()
        assert np.abs(g - r).max() <= 2e-3 * scale + 1e-6, f"parameter {k}: {g} vs {r}"


def test_interior_tiles_against_the_reference():
    """Pictures of 96 x 160: most tiles of the dual step's adjoint have their halos inside the
    picture (the kernel's path without bounds tests), beside the edge tiles."""
    problem, clean, base = _case(iterations=12, every=5, rows=96, columns=160)
    out, _, grads = _device_loss_and_grads(problem, clean, base)
    ref_out, ref_grads = _reference_grads(problem, clean, base)
    got = out.double().cpu().numpy()
    assert np.linalg.norm(got - ref_out) / np.linalg.norm(ref_out) <= 1e-5
    for k, (g, r) in enumerate(zip(grads, ref_grads)):
        scale = np.abs(r).max()
        assert np.abs(g - r).max() <= 2e-3 * scale + 1e-6, f"parameter {k}: {g} vs {r}"


def test_gradients_against_finite_differences():
    from unround.unrolled import unrolled_tgv

    problem, clean, base = _case(iterations=12, every=4, pictures=2)
    _, _, grads = _device_loss_and_grads(problem, clean, base)

    def loss(values):
        with torch.no_grad():
            params = [torch.tensor(v, dtype=torch.float32, device="cuda") for v in values]
            out = unrolled_tgv(problem, *params)
            return torch.mean((out.double() - clean.double()) ** 2).item()

    h = 1e-3
    for k in range(4):
        for n in range(2):
            plus = [b.copy() for b in base]
            minus = [b.copy() for b in base]
            plus[k][n] += h
            minus[k][n] -= h
            fd = (loss(plus) - loss(minus)) / (2 * h)
            # Kinks of the clips and projections within the step, and binary32 in the map.
            assert abs(grads[k][n] - fd) <= 8e-2 * abs(fd) + 1e-4, f"parameter {k}, picture {n}: {grads[k][n]} vs {fd}"


def test_checkpoint_spacing_does_not_change_the_gradients():
    from unround.unrolled import UnrolledProblem

    problem, clean, base = _case(iterations=15, every=15)
    _, loss0, grads0 = _device_loss_and_grads(problem, clean, base)
    for every in (1, 4, 7):
        other = UnrolledProblem.__new__(UnrolledProblem)
        other.__dict__.update(problem.__dict__)
        from unround.unrolled import _Problem

        other.checkpoint_every = every
        other._raw = _Problem(*[getattr(problem._raw, name) for name, _ in _Problem._fields_])
        other._raw.checkpoint_every = every
        other.checkpoint_floats = int(problem._library.unround_b200_unrolled_checkpoint_floats(other._raw))
        other.workspace_floats = int(problem._library.unround_b200_unrolled_workspace_floats(other._raw))
        _, loss1, grads1 = _device_loss_and_grads(other, clean, base)
        assert loss1 == loss0
        for g0, g1 in zip(grads0, grads1):
            np.testing.assert_allclose(g1, g0, rtol=1e-6, atol=1e-9)
