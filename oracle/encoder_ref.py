"""FP64 CPU reference of the trajectory encoder (TEST INFRASTRUCTURE ONLY).

The same network as the CUDA kernels (tsm_enc_* of the library), written with
PyTorch float64 ops on the CPU so that autograd gives the gradients the
kernels must reproduce:
  conv   relu(conv1d(x, W1, b1, padding=2))        64 channels, k=5
  GRU    r, z, n gates (order r, z, n), hidden 128, one step per point
  head   e = [Wo h_last + bo | exp(u_k) * r_k], r_k = point round(k (n - 1) / 15)
         (halves up, k < 16), normalised, 0 for an empty trajectory; u_k are the
         stored skip log-weights
  loss   mean_p (||e_a - e_b||_2 - y_p)^2
Conv and GRU weights are taken at their BF16-rounded values (as the kernels
use them); the head is FP32.  Gradients are with respect to those values.
Only tests/ imports this module.
"""
from __future__ import annotations

import numpy as np
import torch

NS = 16
SIZES = [("conv_w", (64, 2, 5)), ("conv_b", (64,)), ("w_ih", (384, 64)), ("b_ih", (384,)),
         ("w_hh", (384, 128)), ("b_hh", (384,)), ("w_o", (128, 128)), ("b_o", (128,)), ("skip_scale", (NS,))]
BF16 = {"conv_w", "w_ih", "w_hh"}


def unpack(params: np.ndarray):
    """Flat float32 parameters -> dict of float64 leaf tensors (BF16-rounded
    where the kernels round)."""
    p = torch.from_numpy(np.asarray(params, dtype=np.float32))
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        t = p[o:o + n].reshape(shape)
        if name in BF16:
            t = t.to(torch.bfloat16)
        out[name] = t.to(torch.float64).clone().requires_grad_(True)
        o += n
    assert o == p.numel()
    return out


def _bf16(x):
    return x.to(torch.float32).to(torch.bfloat16).to(torch.float64)


def embed(W, trajs, nrm, bf16_operands=False):
    """bf16_operands: a_t and h_t enter the gate products rounded to BF16, as
    in the tensor-core inference kernel (tsm_enc_embed)."""
    embs = []
    mean = torch.tensor([nrm[0], nrm[1]], dtype=torch.float64)
    inv = torch.tensor([nrm[2], nrm[3]], dtype=torch.float64)
    for t in trajs:
        x = (torch.from_numpy(np.asarray(t, dtype=np.float32)).to(torch.float64) - mean) * inv  # [n, 2]
        n = x.shape[0]
        h = torch.zeros(128, dtype=torch.float64)
        if n > 0:
            a = torch.relu(torch.nn.functional.conv1d(x.T[None], W["conv_w"], W["conv_b"], padding=2))[0].T  # [n, 64]
            for s in range(n):
                ai, hi = (_bf16(a[s]), _bf16(h)) if bf16_operands else (a[s], h)
                gi = W["w_ih"] @ ai + W["b_ih"]
                gh = W["w_hh"] @ hi + W["b_hh"]
                r = torch.sigmoid(gi[:128] + gh[:128])
                z = torch.sigmoid(gi[128:256] + gh[128:256])
                nn_ = torch.tanh(gi[256:] + r * gh[256:])
                h = (1 - z) * nn_ + z * h
        if n > 0:
            idx = [(2 * k * (n - 1) + NS - 1) // (2 * (NS - 1)) for k in range(NS)]
            r = (torch.exp(W["skip_scale"])[:, None] * x[idx]).reshape(-1)
        else:
            r = W["skip_scale"].repeat_interleave(2) * 0.0
        embs.append(torch.cat([W["w_o"] @ h + W["b_o"], r]))
    return torch.stack(embs)


def loss_grad(params, trajs, nrm, ia, ib, y, w=None):
    """-> (loss float, grad float64 [n_params] in the flat layout, pred [P]);
    w: per-pair loss weights (None = 1)."""
    W = unpack(params)
    e = embed(W, trajs, nrm)
    d = e[torch.as_tensor(ia)] - e[torch.as_tensor(ib)]
    pred = torch.linalg.vector_norm(d, dim=1)
    sq = (pred - torch.as_tensor(np.asarray(y), dtype=torch.float64)) ** 2
    if w is not None:
        sq = sq * torch.as_tensor(np.asarray(w, dtype=np.float32), dtype=torch.float64)
    loss = sq.mean()
    loss.backward()
    g = torch.cat([W[name].grad.reshape(-1) for name, _ in SIZES])
    return float(loss.item()), g.numpy(), pred.detach().numpy()
