"""The FP64 CPU reference of the unrolled TGV solve (oracle/unrolled_torch.py), without a GPU:
its forward map against the reference's own C++ solver after the same iterations at the same
parameters, and its autograd gradient against central finite differences (h = 1e-3)."""

import numpy as np
import pytest
import torch

from oracle import reference


def _problem(images, options, iterations):
    from unround.unrolled import UnrolledProblem

    return UnrolledProblem(images, options, iterations=iterations, checkpoint_every=5, device="cpu")


@pytest.mark.skipif(not reference.available(), reason="oracle/_ref is not built")
@pytest.mark.parametrize("iterations", [1, 2, 12])
def test_forward_against_the_reference_solver(iterations):
    from unround import synthetic
    from unround.unrolled import UnrolledProblem  # noqa: F401
    from oracle.unrolled_torch import Reference

    options = ["--method", "tgv", "--alpha1", "1.25", "--alpha0", "2.5", "--iterations", str(iterations),
               "--tolerance", "0", "--record-every", "0"]
    pictures = [synthetic.grey(32, 40, quality=30, seed=s, noise=2).image for s in (1, 2)]
    problem = _problem(pictures, options, iterations)
    ref = Reference(problem)
    ones = torch.ones(2, dtype=torch.float64)
    out = ref.run(2.5 * ones, 1.25 * ones, problem.tau * ones, problem.sigma * ones, iterations).numpy()
    for n, image in enumerate(pictures):
        c = image.components[0]
        solved = reference.solve(image.height, image.width, int(image.color_space),
                                 [(c.coefficients, c.quant_table.reshape(64), c.h_samp_factor, c.v_samp_factor)],
                                 options)
        canvas = solved.canvas.reshape(out.shape[1:])
        assert np.abs(out[n] - canvas).max() <= 1e-9 * np.abs(canvas).max()


def test_autograd_against_finite_differences():
    from unround import synthetic
    from oracle.unrolled_torch import Reference

    options = ["--method", "tgv", "--alpha1", "1", "--alpha0", "2"]
    made = [synthetic.grey(24, 32, quality=30, seed=s, noise=2) for s in (3, 4)]
    problem = _problem([m.image for m in made], options, 8)
    ref = Reference(problem)
    clean = torch.tensor(np.stack([m.samples for m in made]), dtype=torch.float64)
    params = [torch.tensor([2.0, 1.6], dtype=torch.float64), torch.tensor([1.0, 0.8], dtype=torch.float64),
              torch.tensor([problem.tau, 0.9 * problem.tau], dtype=torch.float64),
              torch.tensor([problem.sigma, 1.1 * problem.sigma], dtype=torch.float64)]

    def loss(values):
        return torch.mean((ref.run(*values, 8) - clean) ** 2)

    leaves = [p.clone().requires_grad_(True) for p in params]
    loss(leaves).backward()
    # The map is piecewise smooth (clips, projections): a difference of step 1e-3 straddles some
    # of its kinks (within 5% here), one of step 1e-6 none (within 1e-6).
    for h, tolerance in ((1e-3, 5e-2), (1e-6, 1e-6)):
        for k, leaf in enumerate(leaves):
            for n in range(2):
                plus = [p.clone() for p in params]
                minus = [p.clone() for p in params]
                plus[k][n] += h
                minus[k][n] -= h
                fd = (loss(plus) - loss(minus)).item() / (2 * h)
                g = leaf.grad[n].item()
                assert abs(g - fd) <= tolerance * abs(fd) + 1e-7, f"h {h}, parameter {k}, picture {n}: {g} vs {fd}"
