"""The differentiable unrolled TGV solve (include/unround_b200.h, unround_b200_unrolled_*): a
fixed number of iterations of the method on greyscale pictures from the solver's start, whose
last primal iterate is differentiable with respect to each picture's alpha0, alpha1, tau and
sigma -- for learning the parameters of the reconstruction from pairs of clean pictures and
their JPEG files. The forward pass keeps the state every `checkpoint_every` iterations; the
backward pass recomputes the states between and runs the hand-written adjoint kernels.

    problem = UnrolledProblem(images, settings, iterations=100, checkpoint_every=10)
    x = unrolled_tgv(problem, alpha0, alpha1, tau, sigma)      # (pictures, rows, columns)
    torch.nn.functional.mse_loss(x, clean).backward()

alpha0 ... sigma are tensors of one value per picture on the GPU. The iteration is the
solver's (tgv, relaxation rho); a slack's cost (--slack-cost) is not taken.
"""

from __future__ import annotations

import ctypes
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import numpy.typing as npt
import torch

from unround import jpegio, native


class _Problem(ctypes.Structure):
    _fields_ = (
        ("images", ctypes.c_uint64),
        ("rows", ctypes.c_uint64),
        ("columns", ctypes.c_uint64),
        ("iterations", ctypes.c_uint64),
        ("checkpoint_every", ctypes.c_uint64),
        ("relaxation", ctypes.c_float),
        ("lower", ctypes.c_void_p),
        ("upper", ctypes.c_void_p),
        ("centre", ctypes.c_void_p),
        ("middle", ctypes.c_void_p),
        ("weight", ctypes.c_void_p),
        ("flat_weight", ctypes.c_void_p),
        ("flat", ctypes.c_void_p),
        ("start", ctypes.c_void_p),
    )


def _bind(library: ctypes.CDLL) -> None:
    p, f, d, u64 = ctypes.POINTER(_Problem), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64
    text = (ctypes.c_char_p, ctypes.c_size_t)
    library.unround_b200_unrolled_checkpoint_floats.restype = u64
    library.unround_b200_unrolled_checkpoint_floats.argtypes = [p]
    library.unround_b200_unrolled_workspace_floats.restype = u64
    library.unround_b200_unrolled_workspace_floats.argtypes = [p]
    library.unround_b200_unrolled_forward.restype = ctypes.c_int32
    library.unround_b200_unrolled_forward.argtypes = [p, f, f, f, f, f, f, f, ctypes.c_void_p, *text]
    library.unround_b200_unrolled_backward.restype = ctypes.c_int32
    library.unround_b200_unrolled_backward.argtypes = [p, f, f, f, f, f, f, f, d, ctypes.c_void_p, *text]


def dct_matrix() -> npt.NDArray[np.float64]:
    """C[k][n] of the orthonormal 8-point DCT-II."""
    k = np.arange(8)[:, None]
    n = np.arange(8)[None, :]
    c = 0.5 * np.cos(np.pi * (2 * n + 1) * k / 16)
    c[0, :] = np.sqrt(1 / 8)
    return c


def _blocks_to_canvas(blocks: npt.NDArray[np.float64]) -> npt.NDArray[np.float64]:
    by, bx = blocks.shape[:2]
    return blocks.transpose(0, 2, 1, 3).reshape(by * 8, bx * 8)


class UnrolledProblem:
    """The constants of the unrolled solve of greyscale pictures of one canvas size: each
    coefficient's interval and centre (the DC's centred on its middle), the data term's weights,
    the flat blocks, and the start (the canvas of the clipped centres), from the host model of
    the settings (unround_b200_model); in GPU memory."""

    def __init__(self, images: list[jpegio.Image], settings: list[str] | None = None, *, iterations: int = 100,
                 checkpoint_every: int = 10, relaxation: float = 1.9, device: str | torch.device = "cuda") -> None:
        options = list(settings) if settings is not None else ["--method", "tgv"]
        if not images:
            raise ValueError("a problem has at least one picture")
        c = dct_matrix()
        for image in images:
            if image.color_space != jpegio.ColorSpace.GRAYSCALE or len(image.components) != 1:
                raise ValueError("the unrolled solve takes greyscale pictures")
        shapes = {image.components[0].coefficients.shape[:2] for image in images}
        if len(shapes) != 1:
            raise ValueError("the pictures of a problem have one canvas size")
        shape = next(iter(shapes))
        by, bx = shape

        def constants(image: jpegio.Image) -> tuple:
            # One picture's constants from the host model (the library's calls release the
            # interpreter, so pictures are made on the host's threads at once).
            lower = native.model(image, options, 0, 0).reshape(by, bx, 64)
            upper = native.model(image, options, 0, 1).reshape(by, bx, 64)
            centre = native.model(image, options, 0, 2).reshape(by, bx, 64)
            # The start: the clipped centres' canvas (absolute coefficients).
            zeta = np.clip(centre, lower, upper).reshape(by, bx, 8, 8)
            start = _blocks_to_canvas(np.einsum("vi,abvu,un->abin", c, zeta, c, optimize=True))
            # DC centred on the middle of its interval.
            middle = 0.5 * (lower[..., 0] + upper[..., 0])
            lower, upper, centre = lower.copy(), upper.copy(), centre.copy()
            lower[..., 0] -= middle
            upper[..., 0] -= middle
            centre[..., 0] -= middle
            return (lower, upper, centre, middle / 8.0, native.model(image, options, 0, 4),
                    native.model(image, options, 0, 5), native.model(image, options, 0, 6).reshape(by, bx), start)

        with ThreadPoolExecutor(max_workers=max(1, min(len(images), os.cpu_count() or 1, 16))) as pool:
            made = list(pool.map(constants, images))
        lowers, uppers, centres, middles, weights, flat_weights, flats, starts = (list(x) for x in zip(*made))
        assert shape is not None
        self.images = len(images)
        self.rows, self.columns = shape[0] * 8, shape[1] * 8
        self.iterations = int(iterations)
        self.checkpoint_every = int(checkpoint_every)
        self.relaxation = float(relaxation)
        self.device = torch.device(device)
        # The constants in binary64 on the host, as the model made them.
        self.host = {"lower": np.stack(lowers), "upper": np.stack(uppers), "centre": np.stack(centres),
                     "middle": np.stack(middles), "weight": np.stack(weights), "flat_weight": np.stack(flat_weights),
                     "flat": np.stack(flats), "start": np.stack(starts)}
        as_float = lambda xs: torch.tensor(np.stack(xs), dtype=torch.float32, device=self.device).contiguous()  # noqa: E731
        self.lower = as_float(lowers)
        self.upper = as_float(uppers)
        self.centre = as_float(centres)
        self.middle = as_float(middles)
        self.weight = as_float(weights)
        self.flat_weight = as_float(flat_weights)
        self.flat = torch.tensor(np.stack(flats), dtype=torch.uint8, device=self.device).contiguous()
        self.start = as_float(starts)
        plan = native.model(images[0], options, 0, 7)
        self.tau, self.sigma = float(plan[0]), float(plan[1])
        self._library = native._library()
        _bind(self._library)
        self._raw = _Problem(self.images, self.rows, self.columns, self.iterations, self.checkpoint_every,
                             self.relaxation, self.lower.data_ptr(), self.upper.data_ptr(), self.centre.data_ptr(),
                             self.middle.data_ptr(), self.weight.data_ptr(), self.flat_weight.data_ptr(),
                             self.flat.data_ptr(), self.start.data_ptr())
        self.checkpoint_floats = int(self._library.unround_b200_unrolled_checkpoint_floats(ctypes.byref(self._raw)))
        self.workspace_floats = int(self._library.unround_b200_unrolled_workspace_floats(ctypes.byref(self._raw)))
        if self.checkpoint_floats == 0 or self.workspace_floats == 0:
            raise ValueError("the library refuses the problem's sizes")

    def _params(self, *values: torch.Tensor) -> list[torch.Tensor]:
        out = []
        for v in values:
            v = v.detach().to(device=self.device, dtype=torch.float32).reshape(-1).contiguous()
            if v.numel() != self.images:
                raise ValueError(f"one parameter value per picture ({self.images}), not {v.numel()}")
            out.append(v)
        return out

    def forward(self, alpha0: torch.Tensor, alpha1: torch.Tensor, tau: torch.Tensor, sigma: torch.Tensor
                ) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        """The last primal iterate (pictures, rows, columns), the checkpoints and the workspace."""
        a0, a1, t, s = self._params(alpha0, alpha1, tau, sigma)
        checkpoints = torch.empty(self.checkpoint_floats, dtype=torch.float32, device=self.device)
        workspace = torch.empty(self.workspace_floats, dtype=torch.float32, device=self.device)
        output = torch.empty((self.images, self.rows, self.columns), dtype=torch.float32, device=self.device)
        message = ctypes.create_string_buffer(1024)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        status = self._library.unround_b200_unrolled_forward(
            ctypes.byref(self._raw), a0.data_ptr(), a1.data_ptr(), t.data_ptr(), s.data_ptr(), checkpoints.data_ptr(),
            workspace.data_ptr(), output.data_ptr(), stream, message, 1024)
        native._raise(status, message)
        return output, checkpoints, workspace

    def backward(self, alpha0: torch.Tensor, alpha1: torch.Tensor, tau: torch.Tensor, sigma: torch.Tensor,
                 checkpoints: torch.Tensor, workspace: torch.Tensor, output_grad: torch.Tensor) -> torch.Tensor:
        """The gradients (4, pictures) in binary64: alpha0, alpha1, tau, sigma."""
        a0, a1, t, s = self._params(alpha0, alpha1, tau, sigma)
        grad = output_grad.detach().to(device=self.device, dtype=torch.float32).contiguous()
        grads = torch.empty((4, self.images), dtype=torch.float64, device=self.device)
        message = ctypes.create_string_buffer(1024)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        status = self._library.unround_b200_unrolled_backward(
            ctypes.byref(self._raw), a0.data_ptr(), a1.data_ptr(), t.data_ptr(), s.data_ptr(), checkpoints.data_ptr(),
            workspace.data_ptr(), grad.data_ptr(), grads.data_ptr(), stream, message, 1024)
        native._raise(status, message)
        return grads


class _Unrolled(torch.autograd.Function):
    @staticmethod
    def forward(ctx, problem: UnrolledProblem, alpha0, alpha1, tau, sigma):  # type: ignore[override]
        output, checkpoints, workspace = problem.forward(alpha0, alpha1, tau, sigma)
        ctx.problem = problem
        ctx.save_for_backward(alpha0, alpha1, tau, sigma, checkpoints, workspace)
        return output

    @staticmethod
    def backward(ctx, grad):  # type: ignore[override]
        alpha0, alpha1, tau, sigma, checkpoints, workspace = ctx.saved_tensors
        grads = ctx.problem.backward(alpha0, alpha1, tau, sigma, checkpoints, workspace, grad)
        as_param = [grads[k].to(dtype=p.dtype).reshape(p.shape) for k, p in enumerate((alpha0, alpha1, tau, sigma))]
        return (None, *as_param)


def unrolled_tgv(problem: UnrolledProblem, alpha0: torch.Tensor, alpha1: torch.Tensor, tau: torch.Tensor,
                 sigma: torch.Tensor) -> torch.Tensor:
    """The last primal iterate of the unrolled solve, differentiable with respect to the four
    parameters (one value per picture each)."""
    return _Unrolled.apply(problem, alpha0, alpha1, tau, sigma)


def _main() -> None:
    """One forward and backward pass on seeded synthetic pictures (the bench's pictures: piecewise
    smooth plus noise sigma 2, quality 30), printing the loss and the first picture's gradients:
    a check of the differentiable path on a GPU, and the case its kernels are profiled on."""
    import argparse

    from unround import synthetic

    parser = argparse.ArgumentParser(prog="python -m unround.unrolled")
    parser.add_argument("--pictures", type=int, default=16)
    parser.add_argument("--side", type=int, default=512)
    parser.add_argument("--iterations", type=int, default=20)
    parser.add_argument("--checkpoint-every", type=int, default=10)
    args = parser.parse_args()
    made = [synthetic.grey(args.side, args.side, quality=30, seed=s, noise=2) for s in range(args.pictures)]
    problem = UnrolledProblem([m.image for m in made], ["--method", "tgv", "--alpha1", "1", "--alpha0", "2"],
                              iterations=args.iterations, checkpoint_every=args.checkpoint_every)
    clean = torch.tensor(np.stack([m.samples for m in made]), dtype=torch.float32, device=problem.device)
    leaves = [torch.full((args.pictures,), v, dtype=torch.float32, device=problem.device, requires_grad=True)
              for v in (2.0, 1.0, problem.tau, problem.sigma)]
    loss = torch.mean((unrolled_tgv(problem, *leaves) - clean) ** 2)
    loss.backward()
    print(f"loss {loss.item():.6f}; picture 0: d/d alpha0, alpha1, tau, sigma =",
          [float(leaf.grad[0]) for leaf in leaves])


if __name__ == "__main__":
    _main()
