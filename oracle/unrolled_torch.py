"""Test infrastructure: the FP64 CPU reference of the unrolled TGV solve and its gradient. A
restatement, in torch float64 on the CPU, of N iterations of the reference's TGV primal-dual
method on greyscale pictures (cpp/src/primal_dual.hpp:525-735 the steps; cpp/src/model.cpp:57-72
the proximal map; cpp/src/frames.cpp:401-405 and primal_dual.hpp:401-432 the start), with the
per-picture alpha0, alpha1, tau and sigma as inputs; torch's autograd gives the gradient of a loss
of the last primal iterate with respect to them (the clip's and the projections' derivatives
taken almost everywhere). Its forward map is pinned against the reference's own C++ solver
(oracle/_ref) by the tests. Only tests use it, as the checker of the device's adjoint.

The constants are an UnrolledProblem's (unround.unrolled): each coefficient's interval and
centre with the DC centred on its middle, the middle, the weights, the flat blocks, the start.
"""

from __future__ import annotations

import math

import torch


def _forward_x(f: torch.Tensor) -> torch.Tensor:
    """[j + 1 < W] (f(i, j + 1) - f(i, j)): the forward difference across, 0 in the last column."""
    out = torch.zeros_like(f)
    out[..., :, :-1] = f[..., :, 1:] - f[..., :, :-1]
    return out


def _forward_y(f: torch.Tensor) -> torch.Tensor:
    out = torch.zeros_like(f)
    out[..., :-1, :] = f[..., 1:, :] - f[..., :-1, :]
    return out


def _backward_x(f: torch.Tensor) -> torch.Tensor:
    """[j + 1 < W] f(i, j) - [j > 0] f(i, j - 1): the backward difference of docs/math.md 3.2."""
    out = torch.zeros_like(f)
    out[..., :, :-1] = f[..., :, :-1]
    out[..., :, 1:] = out[..., :, 1:] - f[..., :, :-1]
    return out


def _backward_y(f: torch.Tensor) -> torch.Tensor:
    out = torch.zeros_like(f)
    out[..., :-1, :] = f[..., :-1, :]
    out[..., 1:, :] = out[..., 1:, :] - f[..., :-1, :]
    return out


def _scale(square: torch.Tensor, radius: torch.Tensor) -> torch.Tensor:
    """radius / |q| beyond the ball, 1 within it (cpp/include/unround/operators.hpp:112-116); the
    root is taken only where the ball is left, so that autograd sees no root of 0."""
    outside = square > radius * radius
    norm = torch.sqrt(torch.where(outside, square, torch.ones_like(square)))
    return torch.where(outside, radius / norm, torch.ones_like(square))


def _dct_matrix() -> torch.Tensor:
    k = torch.arange(8, dtype=torch.float64)[:, None]
    n = torch.arange(8, dtype=torch.float64)[None, :]
    c = 0.5 * torch.cos(math.pi * (2 * n + 1) * k / 16)
    c[0, :] = math.sqrt(1 / 8)
    return c


class Reference:
    """The unrolled map in float64 of a problem's constants (moved to the CPU)."""

    def __init__(self, problem, relaxation: float | None = None, dtype: torch.dtype = torch.float64) -> None:
        # The problem's constants as the host model made them (binary64), in `dtype`: float64 is
        # the reference; float32 runs the same map in binary32, which measures how far that
        # arithmetic alone moves the map and its gradient.
        host = {k: torch.from_numpy(v) for k, v in problem.host.items()}
        self.lower = host["lower"].to(dtype)  # (B, by, bx, 64)
        self.upper = host["upper"].to(dtype)
        self.centre = host["centre"].to(dtype)
        self.middle = host["middle"].to(dtype)  # (B, by, bx)
        self.weight = host["weight"].to(dtype)  # (B, 64)
        self.flat_weight = host["flat_weight"].to(dtype)
        self.flat = host["flat"] != 0  # (B, by, bx)
        self.start = host["start"].to(dtype)  # (B, H, W)
        self.rho = problem.relaxation if relaxation is None else relaxation
        self.c = _dct_matrix().to(dtype)

    def _blocks(self, canvas: torch.Tensor) -> torch.Tensor:
        b, h, w = canvas.shape
        return canvas.reshape(b, h // 8, 8, w // 8, 8).permute(0, 1, 3, 2, 4)

    def _canvas(self, blocks: torch.Tensor) -> torch.Tensor:
        b, by, bx = blocks.shape[:3]
        return blocks.permute(0, 1, 3, 2, 4).reshape(b, by * 8, bx * 8)

    def prox(self, v: torch.Tensor, tau: torch.Tensor) -> torch.Tensor:
        """x~ = the canvas of clip((e + t c) / (1 + t), a, b), e the DCT of the block less its middle."""
        c = self.c
        middle = self.middle[..., None, None]
        e = torch.einsum("vi,zabij,uj->zabvu", c, self._blocks(v) - middle, c).reshape(*middle.shape[:3], 64)
        weight = torch.where(self.flat[..., None], self.flat_weight[:, None, None, :], self.weight[:, None, None, :])
        t = tau[:, None, None, None] * weight
        z = torch.clamp((e + t * self.centre) / (1.0 + t), min=self.lower, max=self.upper)
        back = torch.einsum("vi,zabvu,uj->zabij", c, z.reshape(*z.shape[:3], 8, 8), c) + middle
        return self._canvas(back)

    def run(self, alpha0: torch.Tensor, alpha1: torch.Tensor, tau: torch.Tensor, sigma: torch.Tensor,
            iterations: int, checkpoint_every: int = 0) -> torch.Tensor:
        """x~_N of the unrolled solve: P_1, D_1, ..., D_{N-1}, P_N from s_0 = (x0, 0, grad x0, 0).
        checkpoint_every > 0 keeps autograd's tape of only one segment of that many iterations at
        a time (torch.utils.checkpoint recomputes it in the backward pass): the same values and
        gradients in a fraction of the memory, for pictures of 512 x 512 and more."""
        x = self.start.clone()
        zero = torch.zeros_like(x)
        state = (x, zero, zero.clone(), _forward_x(x), _forward_y(x), zero.clone(), zero.clone(), zero.clone())
        params = (alpha0[:, None, None], alpha1[:, None, None], tau[:, None, None], sigma[:, None, None], tau)
        done = 0
        while done < iterations - 1:
            count = iterations - 1 - done if checkpoint_every <= 0 else min(checkpoint_every, iterations - 1 - done)
            if checkpoint_every > 0:
                from torch.utils.checkpoint import checkpoint

                state = checkpoint(self._segment, count, *params, *state, use_reentrant=False)
            else:
                state = self._segment(count, *params, *state)
            done += count
        x, p1, p2 = state[0], state[1], state[2]
        return self.prox(x + params[2] * (_backward_y(p2) + _backward_x(p1)), tau)

    def _segment(self, count: int, a0, a1, tt, ss, tau, x, p1, p2, w1, w2, r11, r22, r12):
        """`count` iterations P_k, D_k from the state s_{k-1}: the state s_{k-1+count}."""
        rho = self.rho
        for _ in range(count):
            v = x + tt * (_backward_y(p2) + _backward_x(p1))
            xt = self.prox(v, tau)
            bar = 2.0 * xt - x
            d1 = _forward_x(r11) + _forward_y(r12)
            d2 = _forward_x(r12) + _forward_y(r22)
            t1 = w1 + tt * (p1 + d1)
            t2 = w2 + tt * (p2 + d2)
            b1 = 2.0 * t1 - w1
            b2 = 2.0 * t2 - w2
            q1 = p1 + ss * (_forward_x(bar) - b1)
            q2 = p2 + ss * (_forward_y(bar) - b2)
            fq = _scale(q1 * q1 + q2 * q2, a1)
            e11 = _backward_x(b1)
            e22 = _backward_y(b2)
            e12 = 0.5 * (_backward_y(b1) + _backward_x(b2))
            s11 = r11 + ss * e11
            s22 = r22 + ss * e22
            s12 = r12 + ss * e12
            fs = _scale(s11 * s11 + s22 * s22 + 2.0 * (s12 * s12), a0)
            x = rho * xt + (1 - rho) * x
            p1, p2 = rho * (q1 * fq) + (1 - rho) * p1, rho * (q2 * fq) + (1 - rho) * p2
            w1, w2 = rho * t1 + (1 - rho) * w1, rho * t2 + (1 - rho) * w2
            r11, r22, r12 = (rho * (s11 * fs) + (1 - rho) * r11, rho * (s22 * fs) + (1 - rho) * r22,
                             rho * (s12 * fs) + (1 - rho) * r12)
        return x, p1, p2, w1, w2, r11, r22, r12
