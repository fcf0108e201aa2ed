"""Error report of the learned-guess network's GPU kernels against the oracle.

Not a test module (pytest does not collect it): a script for profiling and
for reading the error norms the GPU tests bound.  For four networks it runs
the forward pass and the gradients of one batch on the device (tcgen05.mma
GEMMs, planck-refactored_b200/mlp.py) and with oracle/mlp_ref.py, and prints
the relative error norms of the output, the loss and each parameter block.
The first network and batch are those of the first case of
tests/test_mlp_gpu.py (same seeds), so its first three GEMM launches are that
case's forward pass.

    python tests/mlp_error_report.py
"""
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def main():
    import torch

    from oracle import mlp_ref
    M = importlib.import_module("planck-refactored_b200.mlp")
    for dims, n in [([112, 256, 256, 232], 300), ([16, 24, 8], 7), ([40, 64, 32, 48], 130),
                    ([112, 256, 256, 64], 4000)]:
        net = M.MLP(dims, max(n, 512), seed=1)
        rng = np.random.default_rng(2)
        X = rng.normal(size=(n, dims[0])).astype(np.float32)
        T = rng.normal(size=(n, dims[-1])).astype(np.float32)
        Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
        p = net.params()
        Y = net.forward(Xd).cpu().numpy()
        Yo = mlp_ref.forward(dims, p, X)[0]
        g, loss = net.gradients(Xd, Td)
        go, losso = mlp_ref.gradients(dims, p, X, T)
        errs, o = [], 0
        for din, dout in zip(dims[:-1], dims[1:]):
            for size in (din * dout, dout):
                a, b = g[o:o + size], go[o:o + size]
                errs.append(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))
                o += size
        print(dims, n, "fwd rel", np.linalg.norm(Y - Yo) / np.linalg.norm(Yo), "loss rel", abs(loss - losso) / losso,
              "grad rel max", max(errs), [f"{e:.1e}" for e in errs], flush=True)
        net.close()


if __name__ == "__main__":
    main()
