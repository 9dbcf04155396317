"""Parity at the workloads' own sizes and iteration counts, where binary32 drift has the most
room to build up (the reference bounds its own rounding linearly in the iterations,
docs/math.md 9.3): the device against the reference's solver (oracle/_ref, binary64, every host
core) on the same seeded pictures and option strings.

- TGV colour 4032x3024 4:2:0, quality 75, alpha1 = 1, alpha0 = 2, 500 iterations (the bench's
  workload);
- TGV grey with a custom table of steps drawn from 1..64, alpha0 = 3, alpha1 = 1.5, 1000
  iterations, the gap recorded every 50: on a 2048 x 2048 picture of the 8192 x 8192 workload's
  generator (the reference takes about 10 minutes for 8192 x 8192 on 16 cores), every record
  compared;
- four pictures of the 64-picture batched mix (300 iterations, TV and TGV) solved in one
  batch, each against the reference directly;
- the unrolled TGV solve of two 512 x 512 pictures, 100 iterations, checkpoints every 10: the
  forward map and the gradients against the FP64 torch reference (oracle/unrolled_torch.py).

The bar: canvas relative L2 <= 1e-4 and max |difference| <= 2e-3 (0..255), 8-bit output
identical on >= 99.9% of samples, the records' primal values, scaling and partial gap within 1e-4
of the record's scale and their dual values within 1e-2 (the drift binary32 iterates give the
dual value over hundreds of iterations: tests/test_numpy_oracle.py), every coefficient within its
interval in binary64; gradients within 5e-3 of the largest, or within twice the spread that the
same map computed in binary32 on the CPU shows against binary64 where that is more (at 100
iterations the map's kinks make that spread range from 3e-5 to 7e-2 over the four parameters).
The figures are printed in the run's summary."""

import os

import numpy as np
import pytest

from conftest import canvas_figures, report_parity
from oracle import reference
from test_gpu_oracle import MAX_ABS, RECORDS, REL_L2, record_differences, rounded_match

pytestmark = pytest.mark.gpu

DUAL_AFTER_HUNDREDS = 1e-2


def _oracle(image, options):
    components = [(c.coefficients, c.quant_table.reshape(64), c.h_samp_factor, c.v_samp_factor) for c in image.components]
    threads = ["--threads", str(os.cpu_count() or 1)]
    return reference.solve(image.height, image.width, int(image.color_space), components, [*options, *threads])


def _check(name, image, ours, theirs):
    figures = canvas_figures(ours.canvas, theirs.canvas)
    same = rounded_match(ours.picture, theirs.canvas, image)
    worst = record_differences(ours.result.history, theirs.record_iterations, theirs.records)
    inside = all(bool(np.all(c >= p.lower) and np.all(c <= p.upper)) for c, p in zip(ours.coefficients, ours.problems))
    report_parity(name, **figures, same_8bit=same, **{f"record_{k}": v for k, v in worst.items()},
                  inside_intervals=inside)
    assert figures["rel_l2"] <= REL_L2, figures
    assert figures["max_abs"] <= MAX_ABS, figures
    assert same >= 0.999, same
    # The primal value, TGV's scaling and the partial gap within 1e-4 of the record's scale; the
    # dual value after hundreds of iterations within the drift that binary32 iterates give it
    # (about 5e-4 of the scale at 500 iterations in the oracle's binary32 restatement:
    # tests/test_numpy_oracle.py), bounded here by 1e-2.
    assert max(v for k, v in worst.items() if k != "dual") <= RECORDS, worst
    assert worst["dual"] <= DUAL_AFTER_HUNDREDS, worst
    assert inside
    assert ours.result.iterations == theirs.iterations


def test_tgv_colour_4032x3024_500_iterations():
    from unround import native, synthetic

    image = synthetic.colour(3024, 4032, quality=75, seed=0, noise=3.0).image
    options = ["--method", "tgv", "--alpha1", "1", "--alpha0", "2", "--iterations", "500", "--tolerance", "0",
               "--record-every", "100"]
    ours = native.solve(image, options)
    theirs = _oracle(image, options)
    _check("tgv-colour-4032x3024-500it", image, ours, theirs)


def test_tgv_grey_custom_table_1000_iterations():
    from unround import native, synthetic

    image = synthetic.large(2048, seed=5).image
    options = ["--method", "tgv", "--alpha1", "1.5", "--alpha0", "3", "--iterations", "1000", "--tolerance", "0",
               "--record-every", "50"]
    ours = native.solve(image, options)
    theirs = _oracle(image, options)
    gap_ours, gap_theirs = ours.result.history.gap, theirs.records[:, 1] - theirs.records[:, 2]
    samples = image.height * image.width
    report_parity("tgv-grey-2048-custom-1000it gap per sample (device)", **{
        str(int(i)): g / samples for i, g in zip(ours.result.history.iterations[::4], gap_ours[::4])})
    report_parity("tgv-grey-2048-custom-1000it gap per sample (reference)", **{
        str(int(i)): g / samples for i, g in zip(theirs.record_iterations[::4], gap_theirs[::4])})
    _check("tgv-grey-2048-custom-1000it", image, ours, theirs)


def test_batched_mix_pictures_against_the_reference():
    from unround import native, synthetic

    # The mix draws its pictures one after another from one generator: its first eight are the
    # 64-picture mix's first eight. Of them, the two smallest of each method.
    mix = synthetic.mix(8, seed=3, iterations=300)
    chosen = []
    for method in ("tv", "tgv"):
        of_method = sorted((e for e in mix if e.method == method), key=lambda e: e.image.height * e.image.width)
        chosen += of_method[:2]
    assert {e.method for e in chosen} == {"tv", "tgv"}
    decoded, _ = native.solve_batch([e.image for e in chosen], [e.options for e in chosen])
    for entry, ours in zip(chosen, decoded):
        theirs = _oracle(entry.image, entry.options)
        name = (f"mix {entry.method} {'colour' if entry.colour else 'grey'} {entry.image.height}x{entry.image.width}"
                f" q{entry.quality}")
        _check(name, entry.image, ours, theirs)


def test_unrolled_tgv_two_512_pictures_100_iterations():
    import torch

    from oracle.unrolled_torch import Reference
    from unround import synthetic
    from unround.unrolled import UnrolledProblem, unrolled_tgv

    made = [synthetic.grey(512, 512, quality=30, seed=40 + s, noise=2) for s in range(2)]
    problem = UnrolledProblem([m.image for m in made], ["--method", "tgv", "--alpha1", "1", "--alpha0", "2"],
                              iterations=100, checkpoint_every=10)
    clean = np.stack([m.samples for m in made])
    base = [np.array([2.0, 1.6]), np.array([1.0, 0.85]), problem.tau * np.array([1.0, 0.9]),
            problem.sigma * np.array([1.0, 1.1])]
    leaves = [torch.tensor(b, dtype=torch.float32, device="cuda", requires_grad=True) for b in base]
    out = unrolled_tgv(problem, *leaves)
    loss = torch.mean((out.double() - torch.tensor(clean, device="cuda")) ** 2)
    loss.backward()
    grads = [leaf.grad.double().cpu().numpy() for leaf in leaves]

    torch.set_num_threads(os.cpu_count() or 1)

    def reference(dtype):
        ref = Reference(problem, dtype=dtype)
        ref_leaves = [torch.tensor(b, dtype=dtype, requires_grad=True) for b in base]
        ref_out = ref.run(*ref_leaves, problem.iterations, checkpoint_every=10)
        ref_loss = torch.mean((ref_out.double() - torch.tensor(clean)) ** 2)
        ref_loss.backward()
        return ref_out.detach().double(), ref_loss.item(), [leaf.grad.double().numpy() for leaf in ref_leaves]

    ref_out, ref_loss, ref_grads = reference(torch.float64)
    # The same map in binary32 on the CPU: how far binary32 arithmetic alone moves the gradient
    # after 100 iterations of a map with kinks (clips, projections).
    _, _, f32_grads = reference(torch.float32)

    names = ("alpha0", "alpha1", "tau", "sigma")
    figures = canvas_figures(out.detach().double().cpu().numpy(), ref_out.numpy())
    errors = {n: float(np.abs(g - r).max() / np.abs(r).max()) for n, g, r in zip(names, grads, ref_grads)}
    spread = {n: float(np.abs(g - r).max() / np.abs(r).max()) for n, g, r in zip(names, f32_grads, ref_grads)}
    report_parity("unrolled-tgv-2x512-100it-K10", **figures, loss_rel=abs(loss.item() - ref_loss) / ref_loss,
                  **{f"grad_{k}": v for k, v in errors.items()},
                  **{f"binary32_cpu_grad_{k}": v for k, v in spread.items()})
    assert figures["rel_l2"] <= 1e-5, figures
    assert figures["max_abs"] <= MAX_ABS, figures
    # Each gradient within 5e-3 of the largest of its pictures, or within twice what the map in
    # binary32 on the CPU shows, where that is more.
    for name in names:
        assert errors[name] <= max(5e-3, 2.0 * spread[name]), (name, errors, spread, grads, ref_grads)
