"""Times the correction network's tensor-core kernels: forward and backward of the 6-layer periodic
CNN on a batch of B coarse states (the training configuration: B = 64, 64 x 64).

  python neural-pde-surrogate_b200/profile_correction.py [--batch 64] [--n 64] [--iters 50]

Prints per-pass times and the achieved BF16 tensor throughput (2 * MACs of the convolutions / time).
"""
import argparse
import importlib
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))


def conv_macs(B, H, W):
    corr = importlib.import_module("neural-pde-surrogate_b200.correction")
    return sum(B * H * W * co * ci * 9 for ci, co, _, _ in corr.LAYERS)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--iters", type=int, default=50)
    a = ap.parse_args()
    import torch
    corr = importlib.import_module("neural-pde-surrogate_b200.correction")
    ic = importlib.import_module("neural-pde-surrogate_b200.ic")
    B, n = a.batch, a.n
    rng = np.random.default_rng(0)
    net = corr.CorrectionNet(B, n, n, params=rng.normal(0, 0.05, corr.param_count()).astype(np.float32))
    U = torch.stack([torch.from_numpy(ic.to_conserved(*ic.sample("riemann", k, n)[:4])) for k in range(B)]).cuda()
    stats = torch.tensor([1.0, 0.0, 0.0, 2.5, 1.0, 1.0, 1.0, 0.3], dtype=torch.float64, device="cuda")
    net.forward(U, stats)
    net.dout16.copy_(torch.randn_like(net.dout16, dtype=torch.float32).to(torch.bfloat16) * 1e-3)
    net.backward()
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record()
    for _ in range(a.iters):
        net.forward(U, stats)
    e[1].record()
    for _ in range(a.iters):
        net.backward()
    e[2].record()
    torch.cuda.synchronize()
    net.check_device_error()
    fwd = e[0].elapsed_time(e[1]) / a.iters
    bwd = e[1].elapsed_time(e[2]) / a.iters
    macs = conv_macs(B, n, n)
    print(f"batch {B} x {n}^2: forward {fwd * 1e3:.1f} us ({2 * macs / (fwd * 1e-3) / 1e12:.1f} TFLOP/s), "
          f"backward {bwd * 1e3:.1f} us ({4 * macs / (bwd * 1e-3) / 1e12:.1f} TFLOP/s, data + weight gradients)")


if __name__ == "__main__":
    main()
