"""CPU FP64 restatement of the learned step proposal's network, the oracle of its forward pass and gradients.
TEST INFRASTRUCTURE ONLY (tests/ use it as the checker).

The device computes in BF16 operands with FP32 accumulation, rounding to BF16 at the points this restatement
rounds: the inputs, the weights W1, W2, W3, and the activations after each ReLU. Everything else here is FP64:
the products, their sums, the biases and, in the backward pass, every gradient (the rounding points pass gradients
through unchanged, as the device's do). Parameter layout: W1 [16 in][64 out], b1 [64], W2 [64 in][64 out], b2 [64],
W3 [64], b3.
"""
from __future__ import annotations

import numpy as np
import torch

LAYOUT = {"W1": (0, (16, 64)), "b1": (1024, (64,)), "W2": (1088, (64, 64)), "b2": (5184, (64,)),
          "W3": (5248, (64,)), "b3": (5312, (1,))}


def bf16_bits_to_f64(bits: np.ndarray) -> torch.Tensor:
    u = np.asarray(bits, np.uint16).astype(np.uint32) << 16
    return torch.from_numpy(u.view(np.float32).astype(np.float64))


def round_bf16(t: torch.Tensor) -> torch.Tensor:
    """Rounds to BF16 (nearest even) in value, with the gradient passing through."""
    r = t.detach().to(torch.float32).to(torch.bfloat16).to(torch.float64)
    return t + (r - t).detach()


def forward(params: np.ndarray, x_bits: np.ndarray, requires_grad: bool = False):
    """(y, parameter tensors) for BF16 input rows x_bits (n, 16) and FP32 parameters."""
    p = torch.from_numpy(np.asarray(params, np.float32).astype(np.float64))
    if requires_grad:
        p.requires_grad_(True)
    t = {k: p[off:off + int(np.prod(shape))].reshape(shape) for k, (off, shape) in LAYOUT.items()}
    x = bf16_bits_to_f64(x_bits)
    h1 = round_bf16(torch.relu(x @ round_bf16(t["W1"]) + t["b1"]))
    h2 = round_bf16(torch.relu(h1 @ round_bf16(t["W2"]) + t["b2"]))
    y = h2 @ round_bf16(t["W3"]) + t["b3"][0]
    return y, p


def gradient(params: np.ndarray, x_bits: np.ndarray, target: np.ndarray) -> tuple[np.ndarray, float]:
    """dL/dparams and L for L = sum (y - target)^2 / (2 n)."""
    y, p = forward(params, x_bits, requires_grad=True)
    tg = torch.from_numpy(np.asarray(target, np.float32).astype(np.float64))
    loss = ((y - tg) ** 2).sum() / (2 * len(tg))
    loss.backward()
    return p.grad.numpy().copy(), float(loss.detach())
