"""The tcgen05 MLP of the learned PPE warm start, through its C ABI entries.

Bar (written into each assert):
* forward vs a plain PyTorch FP32 evaluation of the same network on the
  same BF16-rounded inputs and weights: rel. L2 <= 1e-3 (BF16 rounding of
  the hidden activation at FP32 rounding ties);
* forward vs the FP64 oracle (oracle/mlp_oracle.py): rel. L2 <= 1e-3;
* gradient vs the FP64 oracle, which rounds to BF16 where the kernels do:
  rel. L2 <= 5e-3 per parameter block; loss terms within 1e-4.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import mlp_oracle as MO

pytestmark = pytest.mark.gpu


def _lib():
    from fluidized_bed_master_b200.engine import lib

    L = lib()
    L.sphdem_mlp_param_count.restype = C.c_int32
    L.sphdem_mlp_forward.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    L.sphdem_mlp_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_double,
                                  C.c_void_p, C.c_void_p]
    return L


def _case(n, seed):
    rng = np.random.default_rng(seed)
    p = MO.init_params(seed)
    p[MO.OFF_B1:MO.OFF_W2] = 0.1 * rng.standard_normal(MO.N_H)
    p[MO.OFF_B2:MO.OFF_W3] = 0.1 * rng.standard_normal(MO.N_H)
    p[MO.OFF_B3] = 0.05
    x = MO.bf16(rng.standard_normal((n, MO.N_IN)))
    t = rng.standard_normal(n)
    w = (rng.uniform(size=n) > 0.2).astype(np.float64)
    return p, x, t, w


def _dev(a, dtype):
    import torch

    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _feat_dev(x):
    import torch

    bits = MO.bf16_bits(x).view(np.int16)
    return torch.tensor(bits, dtype=torch.int16, device="cuda").view(torch.bfloat16)


def _forward_gpu(L, p, x):
    import torch

    n = x.shape[0]
    f = _feat_dev(x)
    pd = _dev(p, torch.float32)
    out = torch.zeros(max(n, 1), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    rc = L.sphdem_mlp_forward(C.c_void_p(f.data_ptr()), n, C.c_void_p(pd.data_ptr()), C.c_void_p(out.data_ptr()),
                              C.c_void_p(st))
    assert rc == 0, rc
    return out.cpu().numpy()[:n].astype(np.float64)


def _torch_reference(p, x):
    """Plain PyTorch FP32 of the same network (BF16-rounded weights and H1)."""
    import torch

    W1, b1, W2, b2, w3, b3 = MO.unpack(p)
    t = lambda a: torch.tensor(np.asarray(a), dtype=torch.float32, device="cuda")  # noqa: E731
    xb = t(x)
    z1 = xb @ t(MO.bf16(W1)).T + t(b1)
    h1 = torch.relu(z1).to(torch.bfloat16).to(torch.float32)
    z2 = h1 @ t(MO.bf16(W2)).T + t(b2)
    y = torch.relu(z2) @ t(MO.bf16(w3)) + float(b3)
    return y.cpu().numpy().astype(np.float64)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("n", [1000, 70001])
def test_forward_matches_torch_fp32_and_oracle(n):
    L = _lib()
    assert L.sphdem_mlp_param_count() == MO.N_PARAM
    p, x, _, _ = _case(n, seed=n)
    y = _forward_gpu(L, p, x)
    assert _rel(y, _torch_reference(p, x)) <= 1e-3
    yo, _ = MO.forward(p, x)
    assert _rel(y, yo) <= 1e-3


@pytest.mark.parametrize("n", [1000, 70001])
def test_gradient_matches_oracle(n):
    import torch

    L = _lib()
    p, x, t, w = _case(n, seed=n + 7)
    ws = float(w.sum())
    g = torch.zeros(MO.N_PARAM + 2, dtype=torch.float32, device="cuda")
    f = _feat_dev(x)
    td, wd, pd = _dev(t, torch.float32), _dev(w, torch.float32), _dev(p, torch.float32)
    st = torch.cuda.current_stream().cuda_stream
    rc = L.sphdem_mlp_grad(C.c_void_p(f.data_ptr()), C.c_void_p(td.data_ptr()), C.c_void_p(wd.data_ptr()), n,
                           C.c_void_p(pd.data_ptr()), ws, C.c_void_p(g.data_ptr()), C.c_void_p(st))
    assert rc == 0, rc
    g = g.cpu().numpy().astype(np.float64)
    go, loss_o, ws_o = MO.grad(p, x, t, w, ws)
    blocks = {"W1": (MO.OFF_W1, MO.OFF_B1), "b1": (MO.OFF_B1, MO.OFF_W2), "W2": (MO.OFF_W2, MO.OFF_B2),
              "b2": (MO.OFF_B2, MO.OFF_W3), "w3": (MO.OFF_W3, MO.OFF_B3), "b3": (MO.OFF_B3, MO.N_PARAM)}
    bad = {k: _rel(g[a:b], go[a:b]) for k, (a, b) in blocks.items()}
    assert all(v <= 5e-3 for v in bad.values()), bad
    assert abs(g[MO.N_PARAM] - loss_o) <= 1e-4 * loss_o
    assert abs(g[MO.N_PARAM + 1] - ws_o) <= 1e-6 * ws_o
