"""Float64 CPU restatement of the schedule GNN -- TEST INFRASTRUCTURE ONLY.

The checker for the library's hand-written GNN kernels (tessera_b200/csrc/gnn.cu): same
architecture, same flat parameter layout (GnnLayout::build), same node features and loss,
evaluated in float64 with torch autograd on the CPU, so that the GPU forward outputs and
backward gradients can be compared element by element.  Only tests import it.
"""
from __future__ import annotations

import numpy as np
import torch


def layout(H: int, L: int, K: int, F: int = 4):
    """Offsets of every parameter block in the flat vector (GnnLayout::build order)."""
    off = {}
    o = 0

    def take(name, n):
        nonlocal o
        off[name] = (o, n)
        o += n

    take("We", H * F)
    take("be", H)
    for l in range(L):
        take(f"W1_{l}", H * (H + 1))
        take(f"b1_{l}", H)
        take(f"W2_{l}", H * 2 * H)
        take(f"b2_{l}", H)
    take("wn", H)
    take("bn", 1)
    take("Wg1", H * H)
    take("bg1", H)
    take("Wg2", (K - 1) * H)
    take("bg2", K - 1)
    return off, o


def graph_batch(problems):
    """Node features [h, sum|J|/4, sum J/4, 1], both directions of every edge, node offsets."""
    feats, src, dst, w, goff = [], [], [], [], [0]
    base = 0
    for p in problems:
        n = p.n
        sa = np.zeros(n)
        ss = np.zeros(n)
        for i, j, x in zip(p.ei, p.ej, p.ew):
            if i == j:
                continue
            sa[i] += abs(x); sa[j] += abs(x); ss[i] += x; ss[j] += x
            src += [base + i, base + j]; dst += [base + j, base + i]; w += [x, x]
        feats.append(np.stack([p.h, sa / 4, ss / 4, np.ones(n)], axis=1))
        base += n
        goff.append(base)
    return (torch.tensor(np.concatenate(feats), dtype=torch.float64), torch.tensor(src, dtype=torch.long),
            torch.tensor(dst, dtype=torch.long), torch.tensor(w, dtype=torch.float64), goff)


def forward(theta: torch.Tensor, problems, H: int, L: int, K: int):
    off, _ = layout(H, L, K)

    def P(name, shape):
        o, n = off[name]
        return theta[o:o + n].reshape(shape)

    feat, src, dst, w, goff = graph_batch(problems)
    Nn = feat.shape[0]
    x = torch.relu(feat @ P("We", (H, 4)).T + P("be", (H,)))
    for l in range(L):
        inp = torch.cat([x[src], w[:, None]], dim=1)
        m = torch.relu(inp @ P(f"W1_{l}", (H, H + 1)).T + P(f"b1_{l}", (H,)))
        a = torch.zeros(Nn, H, dtype=torch.float64).index_add(0, dst, m)
        u = torch.cat([x, a], dim=1) @ P(f"W2_{l}", (H, 2 * H)).T + P(f"b2_{l}", (H,))
        x = x + torch.relu(u)
    p = torch.sigmoid(x @ P("wn", (H,)) + P("bn", (1,)))
    knots = []
    for g in range(len(problems)):
        gm = x[goff[g]:goff[g + 1]].mean(dim=0)
        z = torch.relu(P("Wg1", (H, H)) @ gm + P("bg1", (H,)))
        o = P("Wg2", (K - 1, H)) @ z + P("bg2", (K - 1,))
        d = torch.nn.functional.softplus(o)
        c = torch.cat([torch.zeros(1, dtype=torch.float64), torch.cumsum(d, 0)])
        knots.append(c / c[-1])
    return torch.stack(knots), p


def loss_and_grad(params: np.ndarray, problems, target_knots, target_spins, H, L, K, lk, ln):
    theta = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    knots, p = forward(theta, problems, H, L, K)
    tk = torch.tensor(np.asarray(target_knots).reshape(knots.shape), dtype=torch.float64)
    ts = torch.tensor(np.asarray(target_spins), dtype=torch.float64)
    lab = ts >= 0
    loss = lk * ((knots - tk) ** 2).mean()
    if lab.any():
        q = p[lab].clamp(1e-7, 1 - 1e-7)
        loss = loss + ln * (-(ts[lab] * torch.log(q) + (1 - ts[lab]) * torch.log(1 - q))).mean()
    loss.backward()
    return float(loss.detach()), theta.grad.numpy().copy(), knots.detach().numpy(), p.detach().numpy()
