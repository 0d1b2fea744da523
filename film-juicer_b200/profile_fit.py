"""Runs the fitting chain's forward and adjoint once each on the differentiation
workload (16 seeded 512 x 512 crops stacked into one 8192 x 512 image), for a
single-kernel ncu capture of fjb_fit_forward / fjb_fit_vjp:

    python film-juicer_b200/profile_fit.py --route print
"""
from __future__ import annotations

import argparse
import os
import sys


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--route", choices=("direct", "print"), default="print")
    ap.add_argument("--crops", type=int, default=16)
    ap.add_argument("--size", type=int, default=512)
    args = ap.parse_args(argv)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    import __graft_entry__

    __graft_entry__.package()
    import numpy as np
    import torch

    from film_juicer_b200 import fitting, prepare, runtime

    rec = prepare.HostRecord(prepare.PreparedRecipe.load(os.path.join(root, "tests", "golden",
                                                                      f"recipe_{args.route}.npz")))
    dr = runtime.DeviceRecipe(rec)
    src = np.concatenate([prepare.synthetic_frame(args.size, args.size, seed=20261210 + i) for i in range(args.crops)])
    s = torch.from_numpy(np.ascontiguousarray(src)).cuda()
    th = fitting.default_theta(dr)
    out = fitting.forward(dr, th, s)
    g = torch.randn_like(out)
    grad = fitting.vjp(dr, th, s, g)
    torch.cuda.synchronize()
    print("gradient", [round(float(v), 6) for v in grad.cpu()])
    dr.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
